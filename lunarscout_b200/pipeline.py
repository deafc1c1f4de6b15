"""Patch enumeration and the bounded compute -> write pipeline
(mirrors src/lunarscout/_numba_horizon/pipeline.py:27-450).

Patches are row-major 128-pixel tiles of the primary DEM with partial right
and bottom edges kept.  Structurally complete tiles are skipped (resume).
One thread drives the GPU, a second publishes files through a bounded queue,
so at most ``writer_queue_capacity`` computed tiles wait in host memory.
Cancellation is checked between patches (a running kernel is never
interrupted) and the first error stops both threads and is re-raised.
"""

from __future__ import annotations

import queue
import threading
import time
from collections.abc import Callable, Sequence
from dataclasses import dataclass
from pathlib import Path
from typing import Any

from .contract import PATCH_SIZE


class HorizonPipelineCancelled(RuntimeError):
    """Cancellation was observed between bounded pipeline units."""


@dataclass(frozen=True, slots=True)
class PatchDescriptor:
    index: int
    tile_x: int
    tile_y: int
    patch_x: int
    patch_y: int
    width: int
    height: int

    @property
    def kernel_width(self) -> int:
        return PATCH_SIZE

    @property
    def kernel_height(self) -> int:
        return PATCH_SIZE


@dataclass(frozen=True, slots=True)
class HorizonProgress:
    processed_patches: int
    total_patches: int
    percent: float
    stage: str
    message: str
    file_name: str | None = None


@dataclass(frozen=True, slots=True)
class PipelineResult:
    output_paths: tuple[Path, ...]
    skipped_patches: int
    wall_seconds: float
    compute_seconds: float
    write_seconds: float
    maximum_writer_queue_depth: int


def enumerate_patches(width: int, height: int, *,
                      include_partial_edges: bool = True) -> list[PatchDescriptor]:
    """Row-major 128-pixel patches of a width x height grid."""
    if (isinstance(width, bool) or isinstance(height, bool) or not isinstance(width, int)
            or not isinstance(height, int) or width <= 0 or height <= 0):
        raise ValueError("DEM dimensions must be positive integers")
    if not include_partial_edges and (width % PATCH_SIZE or height % PATCH_SIZE):
        raise ValueError("DEM dimensions must be even multiples of 128")
    patches = []
    for patch_y in range((height + PATCH_SIZE - 1) // PATCH_SIZE):
        for patch_x in range((width + PATCH_SIZE - 1) // PATCH_SIZE):
            tile_x, tile_y = patch_x * PATCH_SIZE, patch_y * PATCH_SIZE
            patches.append(PatchDescriptor(len(patches), tile_x, tile_y, patch_x, patch_y,
                                           min(PATCH_SIZE, width - tile_x),
                                           min(PATCH_SIZE, height - tile_y)))
    return patches


def run_bounded_pipeline(
    patches: Sequence[PatchDescriptor],
    *,
    store,
    compute_patch: Callable[[PatchDescriptor], Any],
    write_patch: Callable[[PatchDescriptor, Any], Path],
    observer_elevation_m: float = 0.0,
    skip_existing: bool = True,
    writer_queue_capacity: int = 2,
    progress_callback: Callable[[HorizonProgress], None] | None = None,
    cancellation_requested: Callable[[], bool] | None = None,
) -> PipelineResult:
    """Compute each pending patch and publish it; returns the written paths."""
    if writer_queue_capacity < 1:
        raise ValueError("writer_queue_capacity must be positive")
    started = time.perf_counter()
    cancelled = cancellation_requested or (lambda: False)
    if cancelled():
        raise HorizonPipelineCancelled("Horizon generation was cancelled.")
    pending = []
    skipped = 0
    for patch in patches:
        existing = (store.find_existing_path(patch.tile_y, patch.tile_x, observer_elevation_m)
                    if skip_existing else None)
        if existing is None:
            pending.append(patch)
        else:
            skipped += 1

    def emit(event: HorizonProgress) -> None:
        if progress_callback is not None:
            progress_callback(event)

    total = len(pending)
    emit(HorizonProgress(0, total, 10.0, "prepare_patches", "Preparing horizon patch pipeline."))
    if total == 0:
        emit(HorizonProgress(0, 0, 100.0, "complete", "No horizon patches need to be generated."))
        return PipelineResult((), skipped, time.perf_counter() - started, 0.0, 0.0, 0)
    emit(HorizonProgress(0, total, 15.0, "process_patches", "Starting horizon patch generation."))

    handoff: queue.Queue = queue.Queue(maxsize=writer_queue_capacity)
    done = object()
    stop = threading.Event()
    errors: list[BaseException] = []
    error_lock = threading.Lock()
    paths: list[Path] = []
    stats = {"compute": 0.0, "write": 0.0, "depth": 0, "processed": 0}

    def fail(error: BaseException) -> None:
        with error_lock:
            if not errors:
                errors.append(error)
        stop.set()

    def put(item) -> bool:
        while True:
            try:
                handoff.put(item, timeout=0.05)
                stats["depth"] = max(stats["depth"], handoff.qsize())
                return True
            except queue.Full:
                if stop.is_set():
                    return False

    def writer() -> None:
        while True:
            item = handoff.get()
            try:
                if item is done:
                    return
                if stop.is_set():
                    continue
                patch, payload = item
                try:
                    if cancelled():
                        raise HorizonPipelineCancelled("Horizon generation was cancelled.")
                    t0 = time.perf_counter()
                    path = write_patch(patch, payload)
                    stats["write"] += time.perf_counter() - t0
                    paths.append(path)
                    stats["processed"] += 1
                    n = stats["processed"]
                    emit(HorizonProgress(n, total, n * 100.0 / total, "process_patches",
                                         f"Generated {n}/{total} horizon patches.", path.name))
                except BaseException as error:  # noqa: BLE001 - re-raised by the caller
                    fail(error)
            finally:
                handoff.task_done()

    thread = threading.Thread(target=writer, name="horizon-output-writer", daemon=True)
    thread.start()
    try:
        for patch in pending:
            if stop.is_set():
                break
            if cancelled():
                raise HorizonPipelineCancelled("Horizon generation was cancelled.")
            t0 = time.perf_counter()
            payload = compute_patch(patch)
            stats["compute"] += time.perf_counter() - t0
            if not put((patch, payload)):
                break
    except BaseException as error:  # noqa: BLE001
        fail(error)
    finally:
        while True:
            try:
                handoff.put(done, timeout=0.05)
                break
            except queue.Full:
                continue
        thread.join()
    if errors:
        raise errors[0]
    emit(HorizonProgress(total, total, 100.0, "complete", "Horizons generation complete."))
    return PipelineResult(tuple(paths), skipped, time.perf_counter() - started,
                          stats["compute"], stats["write"], stats["depth"])
