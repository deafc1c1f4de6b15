"""Horizon tile files: naming, completeness, staged writes, and the .cbin codec
on the GPU (mirrors src/lunarscout/_numba_horizon/file_format.py:18-415).

File layout (unchanged from the reference): ``root/{y:05d}/horizon_{y:05d}_
{x:05d}_{dm:03d}.{cbin,bin}`` where ``dm`` is the observer height in
decimetres; ``.bin`` holds little-endian float32 degrees [16384][1440]
(94,371,840 bytes, or +28 for the legacy metadata tail); ``.cbin`` holds per
pixel a u16 length and a delta-coded block.  Writes go to a staging file in
the destination directory, are fsynced and published with ``os.replace``.
"""

from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path
from uuid import uuid4

import numpy as np

from ._native import call, pinned_empty
from .contract import AZIMUTH_COUNT, PATCH_SIZE, PIXEL_COUNT

TOTAL_SAMPLES = PIXEL_COUNT * AZIMUTH_COUNT
RAW_FILE_BYTES = TOTAL_SAMPLES * 4
MAX_COMPRESSED_BLOCK_BYTES = 2 * AZIMUTH_COUNT
MAX_PAYLOAD_BYTES = PIXEL_COUNT * (MAX_COMPRESSED_BLOCK_BYTES + 2)


class TileCodec:
    """.cbin encode/decode on a device (one ls200 context)."""

    def __init__(self, device_id: int = 0, *, context=None):
        from .lightmap_cuda import LightingContext

        self._owner = None
        if context is None:
            self._owner = LightingContext(device_id)
            context = self._owner.handle
        self._context = context
        self._lock = threading.Lock()
        self._payload = pinned_empty(MAX_PAYLOAD_BYTES, np.uint8)

    def close(self) -> None:
        if self._owner is not None:
            self._owner.close()
            self._owner = None

    def encode(self, degrees: np.ndarray) -> bytes:
        values = np.ascontiguousarray(degrees, dtype=np.float32).reshape(-1)
        if values.size != TOTAL_SAMPLES:
            raise ValueError("degrees must hold 16384 x 1440 samples")
        size = ctypes.c_int64()
        with self._lock:
            call("ls200_cbin_encode", self._context, values, self._payload.ctypes.data,
                 MAX_PAYLOAD_BYTES, ctypes.byref(size))
            return bytes(self._payload[: size.value])

    def encode_device(self, device_degrees: int, device_payload: int) -> int:
        size = ctypes.c_int64()
        call("ls200_cbin_encode_device", self._context, ctypes.c_void_p(device_degrees),
             ctypes.c_void_p(device_payload), ctypes.byref(size))
        return int(size.value)

    def decode(self, payload, out: np.ndarray | None = None) -> np.ndarray:
        data = np.frombuffer(payload, dtype=np.uint8)
        if out is None:
            out = np.empty((PIXEL_COUNT, AZIMUTH_COUNT), dtype=np.float32)
        with self._lock:
            call("ls200_cbin_decode", self._context, data.ctypes.data, data.size,
                 out.reshape(-1))
        return out


def normalize_tile(degrees, *, valid_width: int = PATCH_SIZE,
                   valid_height: int = PATCH_SIZE) -> np.ndarray:
    """Full 128x128 pixel-major tile; pixels outside the valid rectangle are
    -50 deg, the codec's minimum (file_format.py:93-120)."""
    if not 1 <= valid_width <= PATCH_SIZE or not 1 <= valid_height <= PATCH_SIZE:
        raise ValueError("valid tile dimensions must be between 1 and 128")
    source = np.asarray(degrees, dtype=np.float32)
    expected = (valid_width * valid_height, AZIMUTH_COUNT)
    full = (PIXEL_COUNT, AZIMUTH_COUNT)
    if source.shape not in (expected, full):
        raise ValueError(f"degrees must have shape {expected} or {full}")
    if np.any(np.isnan(source)):
        raise ValueError("degrees must not contain NaN values")
    if valid_width == PATCH_SIZE and valid_height == PATCH_SIZE:
        return np.ascontiguousarray(source)
    padded = np.full((PATCH_SIZE, PATCH_SIZE, AZIMUTH_COUNT), -50.0, dtype=np.float32)
    if source.shape == full:
        valid = source.reshape(PATCH_SIZE, PATCH_SIZE, AZIMUTH_COUNT)[:valid_height, :valid_width]
    else:
        valid = source.reshape(valid_height, valid_width, AZIMUTH_COUNT)
    padded[:valid_height, :valid_width] = valid
    return padded.reshape(full)


def _staged_write(final_path: Path, chunks) -> Path:
    final_path.parent.mkdir(parents=True, exist_ok=True)
    staging = final_path.parent / f"{final_path.stem}.{uuid4().hex}.tmp{final_path.suffix}"
    try:
        with staging.open("wb", buffering=1024 * 1024) as handle:
            for chunk in chunks:
                handle.write(chunk)
            handle.flush()
            os.fsync(handle.fileno())
        os.replace(staging, final_path)
    except BaseException:
        try:
            staging.unlink(missing_ok=True)
        except OSError:
            pass
        raise
    return final_path


class HorizonTileStore:
    """Tile naming, lookup precedence, completeness and staged publication
    (file_format.py:283-415)."""

    def __init__(self, root_directory, *, read_legacy_flat_files: bool = True,
                 codec: TileCodec | None = None):
        self.root = Path(root_directory)
        if not str(self.root):
            raise ValueError("horizon root directory must be provided")
        self.read_legacy_flat_files = bool(read_legacy_flat_files)
        self.codec = codec

    @staticmethod
    def _elevation_decimeters(observer_elevation_m: float) -> int:
        value = int(float(observer_elevation_m) * 10.0)  # truncates like the C# cast
        if not 0 <= value <= 999:
            raise ValueError("observer elevation must fit the D3 filename field")
        return value

    @staticmethod
    def _coordinate(value: int) -> int:
        if isinstance(value, bool) or not isinstance(value, (int, np.integer)) \
                or not 0 <= int(value) <= 99999:
            raise ValueError("horizon tile coordinates must fit the D5 filename field")
        return int(value)

    def build_file_name(self, tile_y: int, tile_x: int, observer_elevation_m: float, *,
                        compress: bool) -> str:
        y, x = self._coordinate(tile_y), self._coordinate(tile_x)
        dm = self._elevation_decimeters(observer_elevation_m)
        return f"horizon_{y:05d}_{x:05d}_{dm:03d}{'.cbin' if compress else '.bin'}"

    def build_path(self, tile_y: int, tile_x: int, observer_elevation_m: float, *,
                   compress: bool) -> Path:
        name = self.build_file_name(tile_y, tile_x, observer_elevation_m, compress=compress)
        return self.root / f"{int(tile_y):05d}" / name

    def candidate_paths(self, tile_y: int, tile_x: int, observer_elevation_m: float):
        compressed = self.build_file_name(tile_y, tile_x, observer_elevation_m, compress=True)
        raw = self.build_file_name(tile_y, tile_x, observer_elevation_m, compress=False)
        folder = self.root / f"{int(tile_y):05d}"
        candidates = [folder / compressed, folder / raw]
        if self.read_legacy_flat_files:
            candidates += [self.root / compressed, self.root / raw]
        return tuple(candidates)

    @staticmethod
    def is_complete(path) -> bool:
        """Structural completeness: exact .bin size, or exactly 16384
        well-formed .cbin blocks with no trailing bytes."""
        candidate = Path(path)
        try:
            suffix = candidate.suffix.lower()
            if suffix == ".bin":
                return candidate.stat().st_size in (RAW_FILE_BYTES, RAW_FILE_BYTES + 28)
            if suffix != ".cbin" or candidate.stat().st_size <= 0:
                return False
            with candidate.open("rb") as handle:
                for _ in range(PIXEL_COUNT):
                    prefix = handle.read(2)
                    if len(prefix) != 2:
                        return False
                    length = int.from_bytes(prefix, "little")
                    if not 1 <= length <= MAX_COMPRESSED_BLOCK_BYTES:
                        return False
                    if len(handle.read(length)) != length:
                        return False
                return handle.read(1) == b""
        except (OSError, ValueError):
            return False

    def find_existing_path(self, tile_y: int, tile_x: int, observer_elevation_m: float, *,
                           require_complete: bool = True):
        for path in self.candidate_paths(tile_y, tile_x, observer_elevation_m):
            if path.is_file() and (not require_complete or self.is_complete(path)):
                return path
        return None

    def read_path(self, path) -> np.ndarray:
        """float32[128, 128, 1440] degrees of one tile file."""
        candidate = Path(path)
        suffix = candidate.suffix.lower()
        if suffix == ".bin":
            size = candidate.stat().st_size
            if size not in (RAW_FILE_BYTES, RAW_FILE_BYTES + 28):
                raise ValueError("uncompressed horizon file size is invalid")
            with candidate.open("rb") as handle:
                payload = handle.read(RAW_FILE_BYTES)
            values = np.frombuffer(payload, dtype="<f4", count=TOTAL_SAMPLES).astype(np.float32)
        elif suffix == ".cbin":
            if self.codec is None:
                raise ValueError("reading .cbin tiles needs a TileCodec")
            values = self.codec.decode(candidate.read_bytes())
        else:
            raise ValueError("horizon tile must have a .bin or .cbin extension")
        return values.reshape(PATCH_SIZE, PATCH_SIZE, AZIMUTH_COUNT)

    def read(self, tile_y: int, tile_x: int, observer_elevation_m: float):
        path = self.find_existing_path(tile_y, tile_x, observer_elevation_m)
        return None if path is None else self.read_path(path)

    def write(self, tile_y: int, tile_x: int, observer_elevation_m: float, degrees, *,
              compress: bool, valid_width: int = PATCH_SIZE,
              valid_height: int = PATCH_SIZE) -> Path:
        final_path = self.build_path(tile_y, tile_x, observer_elevation_m, compress=compress)
        normalized = normalize_tile(degrees, valid_width=valid_width, valid_height=valid_height)
        if compress:
            if self.codec is None:
                raise ValueError("writing .cbin tiles needs a TileCodec")
            chunks = (self.codec.encode(normalized),)
        else:
            chunks = (normalized.astype("<f4", copy=False).tobytes(order="C"),)
        return _staged_write(final_path, chunks)

    def write_payload(self, tile_y: int, tile_x: int, observer_elevation_m: float,
                      payload, *, compress: bool) -> Path:
        """Publish an already encoded tile (.cbin payload or raw .bin bytes)."""
        final_path = self.build_path(tile_y, tile_x, observer_elevation_m, compress=compress)
        return _staged_write(final_path, (memoryview(payload),))
