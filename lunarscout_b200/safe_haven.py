"""Safe-haven durations per calendar month, fused with the lightmap on the
device (src/lunarscout/_numba_horizon/safe_haven.py and
safe_haven_pipeline.py).

For each pixel and UTC calendar month the product is the longest contiguous
low-Sun run (sun fraction < ``sunlight_threshold``) that overlapped an Earth
outage (Earth margin above the terrain horizon < ``earth_threshold_deg``)
inside that month, in hours; NaN where the month saw no outage, or nothing
but outages.  The month bands and the per-sample band index are host logic
(safe_haven.py:12-72); the fraction, margin and run reduction run in one
device call (``ls200_safe_haven_device``), so neither per-sample stream is
materialised on the host.
"""

from __future__ import annotations

import bisect
from collections.abc import Sequence
from datetime import datetime, timezone

import numpy as np

__all__ = ["month_bands", "month_indices", "safe_haven_patch"]


def _utc(value: datetime | str) -> datetime:
    """A timestamp in UTC (safe_haven.py:12-18): datetimes are converted with
    ``astimezone``; strings are ISO 8601, a trailing ``Z`` meaning UTC."""
    if isinstance(value, datetime):
        return value.astimezone(timezone.utc)
    return datetime.fromisoformat(str(value).replace("Z", "+00:00")).astimezone(timezone.utc)


def month_bands(times_utc: Sequence[datetime | str]) -> tuple[tuple[datetime, datetime], ...]:
    """The calendar months (UTC) that contain any of ``times_utc``, in order,
    as half-open ``(first instant, first instant of the next month)`` pairs
    (safe_haven.py:21-50); empty for no times."""
    months = sorted({(t.year, t.month) for t in map(_utc, times_utc)})
    bands = []
    for year, month in months:
        start = datetime(year, month, 1, tzinfo=timezone.utc)
        stop = datetime(year + month // 12, month % 12 + 1, 1, tzinfo=timezone.utc)
        bands.append((start, stop))
    return tuple(bands)


def month_indices(times_utc: Sequence[datetime | str],
                  bands: Sequence[tuple[datetime, datetime]]) -> np.ndarray:
    """int32 band index of each time, -1 where no band holds it
    (safe_haven.py:53-72).  ``bands`` are sorted, disjoint and half-open, as
    ``month_bands`` returns them."""
    starts = [start for start, _ in bands]
    out = np.full(len(times_utc), -1, dtype=np.int32)
    for i, t in enumerate(map(_utc, times_utc)):
        k = bisect.bisect_right(starts, t) - 1
        if k >= 0 and t < bands[k][1]:
            out[i] = k
    return out


def safe_haven_patch(session, dem, horizons_deg, times_utc, sun_vectors_m, earth_vectors_m, *,
                     tile_y: int, tile_x: int, valid_height: int, valid_width: int,
                     time_step_hours: float, sunlight_threshold: float = 0.2,
                     earth_threshold_deg: float = 2.0):
    """Month bands and the per-band safe-haven durations of one patch
    (safe_haven_pipeline.py:86-96,240-283 for one patch): ``session`` is a
    ``LightmapCudaSession``.  Returns ``(bands, durations)`` with
    ``durations`` a tuple of float32 ``[valid_height, valid_width]`` per
    band."""
    times = tuple(times_utc)
    bands = month_bands(times)
    if not bands:
        raise ValueError("times_utc must span at least one calendar month")
    indices = month_indices(times, bands)
    durations = session.safe_haven_durations(
        dem, horizons_deg, sun_vectors_m, earth_vectors_m, tile_y=tile_y, tile_x=tile_x,
        valid_height=valid_height, valid_width=valid_width, month_index_of=indices,
        band_count=len(bands), time_step_hours=time_step_hours,
        sunlight_threshold=sunlight_threshold, earth_threshold_deg=earth_threshold_deg)
    return bands, durations
