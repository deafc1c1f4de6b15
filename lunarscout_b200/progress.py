"""Progress events of long-running operations (mirrors
src/lunarscout/progress.py:1-27)."""

from __future__ import annotations

from dataclasses import dataclass
from pathlib import Path
from typing import Literal

SelectedBackend = Literal["cpu", "cuda"]


@dataclass(frozen=True, slots=True)
class ProgressEvent:
    """One immutable progress observation."""

    operation: str
    stage: str
    completed: int
    total: int
    fraction: float
    backend: SelectedBackend | None
    message: str
    tile_y: int | None = None
    tile_x: int | None = None
    path: Path | None = None
