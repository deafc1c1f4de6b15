"""The fused horizon -> lighting chain: horizons of a batch of patches are
marched into HBM and every lighting product is evaluated from them there,
with no ``.cbin`` round trip.

The reference computes horizons into tile files (``ls.generate_horizons``)
and its product pipelines read them back per patch
(``nh/lightmap_pipeline.py``, ``nh/psr_pipeline.py:226-253``,
``nh/mission_duration_pipeline.py:69-76``, ``nh/safe_haven_pipeline.py:
240-283``).  ``ProductChain`` keeps the horizons of up to 32 patches on the
device between the persistent multi-site march (``ls200_march_sites``) and
the fused lighting entry points, and can publish the same tiles the
generator writes (device encoder, staged writes) on a writer thread while
the products compute.

Products are evaluated on the marched float32 horizons, with -inf (a ray
that found no terrain sample) read as -50 deg, the value a stored ``.cbin``
tile decodes to there; the PSR session refuses non-finite horizons, and the
lighting signals would turn them into NaN.  A pipeline that reads ``.cbin``
tiles also sees the codec's quantized values (0.0015 deg steps), so products
near a threshold can differ from the file-based chain there.
"""

from __future__ import annotations

import ctypes
import threading
from collections.abc import Sequence
from dataclasses import dataclass

import numpy as np

from . import _native
from .contract import AZIMUTH_COUNT, PATCH_SIZE, PIXEL_COUNT, DemGrid, projection_array
from .lightmap_cuda import DeviceVectors, patch_elevations, validate_vectors

SUBPATCH_SIZE = 8
MAX_BATCH = 32


@dataclass
class PatchBatch:
    """Horizons of a batch of patches resident on the device."""

    patches: list            # PatchDescriptor-like (tile_y, tile_x, height, width)
    horizons: object         # torch float32 [n, 16384, 1440] degrees, -50 outside
    patch_dems: object       # torch float32 [n, 128, 128], zero outside
    geo: np.ndarray          # float64 [n, 6]
    projections: np.ndarray  # float64 [n, 6]
    windows: np.ndarray      # int32 [n, 4] (tile_x, tile_y, valid_width, valid_height)
    lighting_horizons: object = None  # horizons with -inf read as -50 (made on first use)

    def __len__(self) -> int:
        return len(self.patches)


class ProductChain:
    """A device-resident DEM stack (primary first) marching batches of
    patches and evaluating lighting products from the resident horizons.

    ``traversal="exact"`` reproduces the reference's tiles bit for bit;
    ``"ladder"`` is the faster skip-ladder traversal."""

    def __init__(self, dems: Sequence[DemGrid], *, device_id: int = 0,
                 maximum_distance_m: float = 1_000_000.0, observer_elevation_m: float = 0.0,
                 traversal: str = "exact") -> None:
        from .cuda_backend import TRAVERSALS, CudaSession

        if not dems:
            raise ValueError("at least one DEM is required")
        if traversal not in TRAVERSALS:
            raise ValueError(f"traversal must be one of {sorted(TRAVERSALS)}")
        if not np.isfinite(maximum_distance_m) or maximum_distance_m <= 0.0:
            raise ValueError("maximum_distance_m must be finite and positive")
        self.session = CudaSession(device_id)
        self.dems = list(dems)
        self.primary = self.dems[0]
        self.device_dems = [self.session.upload_pyramid(self.session.build_max_pyramid(dem), dem)
                            for dem in self.dems]
        self.maximum_distance_m = float(maximum_distance_m)
        self.observer_elevation_m = float(observer_elevation_m)
        self.traversal = traversal
        self._writer: threading.Thread | None = None
        self._writer_error: BaseException | None = None

    def close(self) -> None:
        self.wait_for_writes()
        for dem in self.device_dems:
            dem.close()
        self.device_dems = []
        self.session.close()

    # -- horizons ---------------------------------------------------------------
    def march(self, patches: Sequence) -> PatchBatch:
        """Horizons (degrees, -50 outside each valid rectangle, as stored
        tiles are padded) of 1 to 32 patches in one persistent launch."""
        import torch

        from .cuda_backend import SiteTile

        patches = list(patches)
        if not 1 <= len(patches) <= MAX_BATCH:
            raise ValueError("a batch holds 1 to 32 patches")
        self.wait_for_writes()
        count = len(patches)
        horizons = torch.empty((count, PIXEL_COUNT, AZIMUTH_COUNT), dtype=torch.float32,
                               device="cuda")
        tiles = [SiteTile(tuple(self.device_dems), p.tile_x, p.tile_y, self.maximum_distance_m,
                          self.observer_elevation_m) for p in patches]
        torch.cuda.synchronize()
        self.session.march_sites(tiles, device_out=horizons.data_ptr(),
                                 azimuth_count=AZIMUTH_COUNT, subpatch_size=SUBPATCH_SIZE,
                                 traversal=self.traversal, degrees=True)
        grid = horizons.view(count, PATCH_SIZE, PATCH_SIZE, AZIMUTH_COUNT)
        for i, p in enumerate(patches):
            if p.width < PATCH_SIZE:
                grid[i, :, p.width:] = -50.0
            if p.height < PATCH_SIZE:
                grid[i, p.height:] = -50.0
        dems = torch.from_numpy(np.stack([
            patch_elevations(self.primary, p.tile_y, p.tile_x, p.height, p.width)
            for p in patches])).cuda()
        geo = np.ascontiguousarray(np.repeat(self.primary.geo_transform[None, :], count, 0),
                                   dtype=np.float64)
        projections = np.ascontiguousarray(
            np.repeat(projection_array(self.primary.projection)[None, :], count, 0))
        windows = np.array([(p.tile_x, p.tile_y, p.width, p.height) for p in patches],
                           dtype=np.int32)
        torch.cuda.synchronize()
        return PatchBatch(patches, horizons, dems, geo, projections, windows)

    def write_tiles(self, batch: PatchBatch, store, *, compress: bool = True,
                    background: bool = True) -> None:
        """Publish the batch's tiles into a ``HorizonTileStore`` (the
        generator's file bytes: device encoder for ``.cbin``).  With
        ``background`` the payloads are copied to the host now and written by
        a thread; the next ``march`` (or ``wait_for_writes``) joins it."""
        import torch

        from .file_format import MAX_PAYLOAD_BYTES, TileCodec

        self.wait_for_writes()
        payloads = []
        if compress:
            codec = TileCodec(context=self.session.context)
            buffer = torch.empty(MAX_PAYLOAD_BYTES, dtype=torch.uint8, device="cuda")
            try:
                for i in range(len(batch)):
                    size = codec.encode_device(batch.horizons[i].data_ptr(), buffer.data_ptr())
                    payloads.append(buffer[:size].cpu().numpy().tobytes())
            finally:
                codec.close()
        else:
            for i in range(len(batch)):
                payloads.append(batch.horizons[i].cpu().numpy().astype("<f4").tobytes())
        jobs = [(p.tile_y, p.tile_x, data) for p, data in zip(batch.patches, payloads)]

        def write():
            try:
                for tile_y, tile_x, data in jobs:
                    store.write_payload(tile_y, tile_x, self.observer_elevation_m, data,
                                        compress=compress)
            except BaseException as error:  # re-raised by wait_for_writes
                self._writer_error = error

        if background:
            self._writer = threading.Thread(target=write, name="horizon-tile-writer",
                                            daemon=True)
            self._writer.start()
        else:
            write()
            self._raise_writer_error()

    def wait_for_writes(self) -> None:
        if self._writer is not None:
            self._writer.join()
            self._writer = None
        self._raise_writer_error()

    def _raise_writer_error(self) -> None:
        if self._writer_error is not None:
            error, self._writer_error = self._writer_error, None
            raise error

    # -- products ---------------------------------------------------------------
    def _lighting_args(self, batch: PatchBatch):
        import torch

        if batch.lighting_horizons is None:
            batch.lighting_horizons = torch.where(torch.isneginf(batch.horizons),
                                                  torch.full_like(batch.horizons, -50.0),
                                                  batch.horizons).contiguous()
            torch.cuda.synchronize()
        return (self.session.context, len(batch), ctypes.c_void_p(batch.patch_dems.data_ptr()),
                batch.geo.ctypes.data, batch.projections.ctypes.data, batch.windows.ctypes.data,
                ctypes.c_void_p(batch.lighting_horizons.data_ptr()))

    def _crop(self, batch: PatchBatch, grid: np.ndarray) -> list:
        """Per patch, the valid rectangle of [n, ..., 16384] planes."""
        shaped = grid.reshape(*grid.shape[:-1], PATCH_SIZE, PATCH_SIZE)
        return [np.ascontiguousarray(shaped[i, ..., :p.height, :p.width])
                for i, p in enumerate(batch.patches)]

    def sun_fraction_bytes(self, batch: PatchBatch, sun_vectors_m):
        """uint8 lightmap bytes int(255 * fraction) of every patch and time
        step, left on the device: torch [n, T, 16384] (lightmap_cuda.py:36-182)."""
        return self._lighting(batch, sun_vectors_m, signal=1)

    def sun_fractions(self, batch: PatchBatch, sun_vectors_m):
        """float32 fractions, torch [n, T, 16384] on the device."""
        return self._lighting(batch, sun_vectors_m, signal=0)

    def _lighting(self, batch: PatchBatch, vectors_m, *, signal: int):
        import torch

        vectors = np.ascontiguousarray(validate_vectors(vectors_m), dtype=np.float32)
        dtype = torch.uint8 if signal == 1 else torch.float32
        out = torch.empty((len(batch), len(vectors), PIXEL_COUNT), dtype=dtype, device="cuda")
        frames = torch.empty(len(batch) * PIXEL_COUNT * 12, dtype=torch.float32, device="cuda")
        table = DeviceVectors(self.session.context, vectors)
        try:
            _native.call("ls200_lighting_device", *self._lighting_args(batch), table.handle, 0,
                         len(vectors), signal, ctypes.c_void_p(frames.data_ptr()),
                         ctypes.c_void_p(out.data_ptr()))
            _native.call("ls200_synchronize", self.session.context)
        finally:
            table.close()
        return out

    def reduced_sun_vectors(self, sun_vectors_m) -> tuple[np.ndarray, np.ndarray]:
        """The PSR product's vector reduction over the primary DEM
        (reduce_sun_vectors_for_psr, psr.py:61-91, on the device), cached
        for the last vector table."""
        from .psr_cuda import reduce_vectors_on

        vectors = np.ascontiguousarray(sun_vectors_m, dtype=np.float64)
        key = (vectors.shape, vectors.tobytes())
        if getattr(self, "_reduction_key", None) != key:
            self._reduction = reduce_vectors_on(self.session.context, self.primary, vectors)
            self._reduction_key = key
        return self._reduction

    def psr(self, batch: PatchBatch, sun_vectors_m, *, reduce: bool = True) -> list:
        """uint8 PSR masks [valid_h, valid_w] per patch: the PSR product of
        psr_pipeline.py:259-263 — the vectors reduced over the primary DEM
        (reduced_sun_vectors), then psr_cuda.py:57-186 on each patch.  With
        ``reduce=False`` the vectors given are used as they are, as
        PsrCudaSession.compute_patch does."""
        import torch

        if reduce:
            sun_vectors_m = self.reduced_sun_vectors(sun_vectors_m)[0]
        vectors = np.ascontiguousarray(validate_vectors(sun_vectors_m), dtype=np.float32)
        out = torch.empty((len(batch), PIXEL_COUNT), dtype=torch.uint8, device="cuda")
        frames = torch.empty(len(batch) * PIXEL_COUNT * 12, dtype=torch.float32, device="cuda")
        table = DeviceVectors(self.session.context, vectors)
        try:
            _native.call("ls200_lighting_device", *self._lighting_args(batch), table.handle, 0,
                         len(vectors), 3, ctypes.c_void_p(frames.data_ptr()),
                         ctypes.c_void_p(out.data_ptr()))
            _native.call("ls200_synchronize", self.session.context)
        finally:
            table.close()
        return self._crop(batch, out.cpu().numpy())

    def mission_durations(self, batch: PatchBatch, sun_vectors_m, *, sample_hours,
                          start_windows, earth_vectors_m=None, sun_threshold: float = 0.5,
                          earth_threshold: float = 0.0, days: bool = False) -> list:
        """float32 [I, valid_h, valid_w] per patch, as
        LightmapCudaSession.mission_durations."""
        import torch

        sun = np.ascontiguousarray(validate_vectors(sun_vectors_m), dtype=np.float32)
        earth = (None if earth_vectors_m is None else
                 np.ascontiguousarray(validate_vectors(earth_vectors_m), dtype=np.float32))
        hours = np.ascontiguousarray(sample_hours, dtype=np.float64)
        if hours.shape != (len(sun),):
            raise ValueError("sample_hours must have one entry per time step")
        windows = np.ascontiguousarray(start_windows, dtype=np.int32).reshape(-1, 2)
        out = torch.empty((len(batch), len(windows), PIXEL_COUNT), dtype=torch.float32,
                          device="cuda")
        sun_table = DeviceVectors(self.session.context, sun)
        earth_table = None if earth is None else DeviceVectors(self.session.context, earth)
        try:
            _native.call("ls200_mission_duration_device", *self._lighting_args(batch),
                         sun_table.handle, None if earth_table is None else earth_table.handle,
                         float(sun_threshold), float(earth_threshold), hours.ctypes.data,
                         windows.ctypes.data, len(windows), 1 if days else 0,
                         ctypes.c_void_p(out.data_ptr()))
        finally:
            sun_table.close()
            if earth_table is not None:
                earth_table.close()
        return self._crop(batch, out.cpu().numpy())

    def safe_haven(self, batch: PatchBatch, sun_vectors_m, earth_vectors_m, *,
                   month_index_of, band_count: int, time_step_hours: float,
                   sunlight_threshold: float = 0.2, earth_threshold_deg: float = 2.0) -> list:
        """float32 [bands, valid_h, valid_w] per patch, as
        LightmapCudaSession.safe_haven_durations."""
        import torch

        sun = np.ascontiguousarray(validate_vectors(sun_vectors_m), dtype=np.float32)
        earth = np.ascontiguousarray(validate_vectors(earth_vectors_m), dtype=np.float32)
        months = np.ascontiguousarray(month_index_of, dtype=np.int32)
        if len(earth) != len(sun) or months.shape != (len(sun),):
            raise ValueError("timestamps, Sun vectors, and Earth vectors must align")
        out = torch.empty((len(batch), int(band_count), PIXEL_COUNT), dtype=torch.float32,
                          device="cuda")
        sun_table = DeviceVectors(self.session.context, sun)
        earth_table = DeviceVectors(self.session.context, earth)
        try:
            _native.call("ls200_safe_haven_device", *self._lighting_args(batch),
                         sun_table.handle, earth_table.handle, float(sunlight_threshold),
                         float(earth_threshold_deg), float(np.float32(time_step_hours)),
                         months.ctypes.data, int(band_count), ctypes.c_void_p(out.data_ptr()))
        finally:
            sun_table.close()
            earth_table.close()
        return self._crop(batch, out.cpu().numpy())

    def earth_visibility(self, batch: PatchBatch, earth_vectors_m, *,
                         threshold_deg: float = 0.0) -> list:
        """float32 [valid_h, valid_w] per patch, as
        LightmapCudaSession.earth_visibility_fraction."""
        import torch

        earth = np.ascontiguousarray(validate_vectors(earth_vectors_m), dtype=np.float32)
        out = torch.empty((len(batch), PIXEL_COUNT), dtype=torch.float32, device="cuda")
        table = DeviceVectors(self.session.context, earth)
        try:
            _native.call("ls200_earth_visibility_device", *self._lighting_args(batch),
                         table.handle, float(threshold_deg), ctypes.c_void_p(out.data_ptr()))
        finally:
            table.close()
        return self._crop(batch, out.cpu().numpy())


__all__ = ["PatchBatch", "ProductChain"]
