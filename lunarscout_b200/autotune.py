"""Autotuner of the persistent multi-site march's launch configuration.

The batched march (``CudaSession.march_sites``) has launch parameters that
change its speed but never its results: how the 32 rays of a warp job are
laid out (L adjacent pixels x 32/L adjacent azimuths: the azimuths per
warp) and the resident blocks per SM (8 blocks at 64
registers, or 6 at 80).  ``tune_batch`` times each candidate on a sample
batch with CUDA events (the march seconds the library reports) and keeps the
fastest; results may be cached per device and workload key in a JSON file.
"""

from __future__ import annotations

import json
import os
from collections.abc import Callable, Sequence
from dataclasses import asdict, dataclass
from pathlib import Path

from .cuda_backend import BatchConfig

#: The default search space: lane layouts x occupancies, the default first.
DEFAULT_CANDIDATES: tuple[BatchConfig, ...] = tuple(
    BatchConfig(lanes, blocks) for lanes in (2, 1, 4, 8, 16, 32) for blocks in (8, 6))


@dataclass(frozen=True, slots=True)
class TuneResult:
    best: BatchConfig
    seconds: dict  # BatchConfig -> best march seconds of the candidate
    key: str | None = None
    cached: bool = False


def select_best(seconds: dict, order: Sequence[BatchConfig]) -> BatchConfig:
    """Fastest candidate; on equal times the earlier one in ``order``."""
    if not seconds:
        raise ValueError("no candidate was timed")
    rank = {config: i for i, config in enumerate(order)}
    return min(seconds, key=lambda c: (seconds[c], rank.get(c, len(rank))))


def workload_key(device_name: str, traversal: str, azimuth_count: int, tile_count: int) -> str:
    return f"{device_name}|{traversal}|az{azimuth_count}|tiles{tile_count}"


def _load_cache(path: Path) -> dict:
    try:
        return json.loads(path.read_text())
    except (OSError, ValueError):
        return {}


def _store_cache(path: Path, key: str, config: BatchConfig) -> None:
    data = _load_cache(path)
    data[key] = asdict(config)
    path.parent.mkdir(parents=True, exist_ok=True)
    staging = path.with_name(f".{path.name}.{os.getpid()}.tmp")
    staging.write_text(json.dumps(data, indent=1, sort_keys=True))
    os.replace(staging, path)


def tune_batch(session, tiles, *, device_out: int, azimuth_count: int = 1440,
               traversal: str = "ladder", candidates: Sequence[BatchConfig] | None = None,
               repeats: int = 1, apply: bool = True, cache_path: str | Path | None = None,
               run: Callable | None = None) -> TuneResult:
    """Time every candidate configuration on ``tiles`` and pick the fastest.

    With ``apply`` the winner is set on the session, otherwise the previous
    configuration is restored.  With ``cache_path`` a stored winner for the
    same device and workload key is used without timing.  ``run`` replaces
    the timed call (``run(session, tiles) -> march seconds``) for tests."""
    if repeats < 1:
        raise ValueError("repeats must be positive")
    order = tuple(candidates or DEFAULT_CANDIDATES)
    key = workload_key(session.info.name, traversal, azimuth_count, len(tiles))
    if cache_path is not None:
        stored = _load_cache(Path(cache_path)).get(key)
        if stored is not None:
            best = BatchConfig(**stored)
            if apply:
                session.set_batch_config(best)
            return TuneResult(best, {}, key, cached=True)

    def default_run(sess, batch):
        return sess.march_sites(batch, device_out=device_out, azimuth_count=azimuth_count,
                                traversal=traversal)[1]

    timed = run or default_run
    previous = session.batch_config()
    seconds = {}
    try:
        for config in order:
            session.set_batch_config(config)
            seconds[config] = min(timed(session, tiles) for _ in range(repeats))
    finally:
        session.set_batch_config(previous)
    best = select_best(seconds, order)
    if apply:
        session.set_batch_config(best)
    if cache_path is not None:
        _store_cache(Path(cache_path), key, best)
    return TuneResult(best, seconds, key)
