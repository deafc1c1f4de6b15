"""CUDA graphs of asynchronous device calls (``ls200_capture_begin`` /
``ls200_capture_end`` in include/ls200.h).

The reference launches each 32-step lighting chunk and waits for it
(``nh/lightmap_cuda.py:226-276``).  Here a whole sequence of chunk launches
is recorded once and replayed with a single ``cudaGraphLaunch``; the recorded
kernels keep reading and writing the same device buffers, so refilling those
buffers and replaying processes the next tile.
"""

from __future__ import annotations

import ctypes
from collections.abc import Callable

from ._native import call, library


class DeviceGraph:
    """An instantiated graph of one context's asynchronous calls."""

    def __init__(self, handle: ctypes.c_void_p):
        self.handle = handle

    @classmethod
    def capture(cls, context, record: Callable[[], None]) -> "DeviceGraph":
        """Run ``record()`` (asynchronous calls on ``context``) in capture mode
        and return the graph of what it issued."""
        call("ls200_capture_begin", context)
        handle = ctypes.c_void_p()
        try:
            record()
        finally:
            # Always leave capture mode; a failed record invalidates the graph.
            status = library().ls200_capture_end(context, ctypes.byref(handle))
        from ._native import check

        check(status, "ls200_capture_end")
        return cls(handle)

    @property
    def nodes(self) -> int:
        count = ctypes.c_int64()
        call("ls200_graph_nodes", self.handle, ctypes.byref(count))
        return int(count.value)

    def launch(self) -> None:
        call("ls200_graph_launch", self.handle)

    def close(self) -> None:
        if self.handle:
            library().ls200_graph_destroy(self.handle)
        self.handle = ctypes.c_void_p()

    def __enter__(self) -> "DeviceGraph":
        return self

    def __exit__(self, *exc) -> None:
        self.close()
