"""DEM adjoint of a time-integrated sun fraction, as a ``torch.autograd.Function``.

No reference counterpart: lunarscout computes horizons and sun fractions but
no derivatives.  The differentiable model (``ls200_sun_loss_forward`` in
``include/ls200.h``) is

    loss = sum over tiles and pixels of w * mean_t F((el_t - h(az_t)) / r),

F the visible fraction of a disk of radius ``r`` above a locally level
horizon line, h the marched horizon interpolated at the sun azimuth as the
reference's margin signal does (``nh/lightmap_cuda.py:125-145``).  The
reference's own fraction (16 slices, 0.27 deg) is piecewise constant in h,
so the smooth F carries the gradient; its radius defaults to 0.2665 deg and
every number made with it is labelled as this model's.

Gradients reach the DEM heights through each ray's winning level-0 sample
(its four bilinear corners and the spherical slope formula) and through the
observer's own terrain height; the march's discrete choices (culling, step
positions, which sample wins) are held fixed, so the gradient is that of the
piecewise-smooth function at the current heights.
"""

from __future__ import annotations

import ctypes
from collections.abc import Sequence

import numpy as np

from ._native import call
from .contract import PATCH_SIZE
from .cuda_backend import TRAVERSALS, SiteTile, site_tile_structs

SMOOTH_DISK_RADIUS_DEG = 0.2665
PLANE = PATCH_SIZE * PATCH_SIZE


class SunLossProblem:
    """A fixed set of tiles, pixel weights and sun vectors over a DEM stack
    whose heights are the differentiable input (one float32 tensor per DEM,
    primary first, each [H, W] on the session's device)."""

    def __init__(self, session, dems: Sequence, tiles: Sequence[tuple[int, int]], weights,
                 sun_vectors, *, maximum_distance_m: float = 20_000.0,
                 observer_elevation_m: float = 0.0, azimuth_count: int = 1440,
                 disk_radius_deg: float = SMOOTH_DISK_RADIUS_DEG, traversal: str = "ladder"):
        import torch

        from .lightmap_cuda import DeviceVectors

        if traversal not in ("exact", "ladder"):
            raise ValueError("traversal must be 'exact' or 'ladder'")
        self.session = session
        self.maximum_distance_m = float(maximum_distance_m)
        self.observer_elevation_m = float(observer_elevation_m)
        self.azimuth_count = int(azimuth_count)
        self.traversal = traversal
        self.disk_radius_deg = float(disk_radius_deg)
        self.device_dems = [session.upload_dem_grid(dem) for dem in dems]
        self.shapes = [(dem.height, dem.width) for dem in dems]
        self.vectors = DeviceVectors(session.context,
                                     np.ascontiguousarray(sun_vectors, dtype=np.float32))
        self.time_count = self.vectors.count
        self.last_seconds = {}
        self.use_tiles(tiles, weights)

    def use_tiles(self, tiles: Sequence[tuple[int, int]], weights) -> None:
        """Replace the tile set (1 to 32 (tile_x, tile_y) origins) and its
        [tiles, 128, 128] pixel weights; DEMs and vectors stay resident."""
        import torch

        if not tiles or len(tiles) > 32:
            raise ValueError("1 to 32 tiles")
        w = torch.as_tensor(np.asarray(weights, dtype=np.float32))
        if w.numel() != len(tiles) * PLANE:
            raise ValueError("weights must hold tile_count x 128 x 128 values")
        self.tiles = [SiteTile(tuple(self.device_dems), int(tx), int(ty),
                               self.maximum_distance_m, self.observer_elevation_m)
                      for tx, ty in tiles]
        self.weights = w.reshape(len(tiles), PLANE).contiguous().cuda()

    def close(self) -> None:
        self.vectors.close()
        for dem in self.device_dems:
            dem.close()

    # -- raw calls -------------------------------------------------------------
    def set_heights(self, heights) -> None:
        import torch

        if len(heights) != len(self.device_dems):
            raise ValueError("one height tensor per DEM of the stack")
        torch.cuda.current_stream().synchronize()
        for dem, shape, h in zip(self.device_dems, self.shapes, heights):
            h = h.detach()
            if tuple(h.shape) != shape:
                raise ValueError(f"heights must have shape {shape}")
            h32 = h.to(device="cuda", dtype=torch.float32).contiguous()
            call("ls200_dem_set_heights_device", dem.handle, ctypes.c_void_p(h32.data_ptr()))

    def forward_value(self, heights=None) -> float:
        """The loss at the given heights (or the DEMs' current ones)."""
        if heights is not None:
            self.set_heights(heights)
        structs, _keep = site_tile_structs(self.tiles)
        loss = ctypes.c_double()
        seconds = np.zeros(2, dtype=np.float64)
        call("ls200_sun_loss_forward", self.session.context,
             ctypes.cast(structs, ctypes.c_void_p), len(self.tiles), self.azimuth_count,
             TRAVERSALS[self.traversal], ctypes.c_void_p(self.weights.data_ptr()),
             self.vectors.handle, self.disk_radius_deg, ctypes.byref(loss), seconds.ctypes.data)
        self.last_seconds["forward_march"] = float(seconds[0])
        self.last_seconds["forward_lighting"] = float(seconds[1])
        return float(loss.value)

    def replay_value(self, heights=None) -> float:
        """The last forward's loss at the given heights with its sampling (the
        march's culling, step positions and winning samples) held fixed; a
        following backward differentiates this function."""
        if heights is not None:
            self.set_heights(heights)
        loss = ctypes.c_double()
        call("ls200_sun_loss_replay", self.session.context, ctypes.byref(loss))
        return float(loss.value)

    def backward_value(self, grad_output: float = 1.0):
        """float64 gradients of grad_output x the last forward's loss."""
        import torch

        grads = [torch.zeros(shape, dtype=torch.float64, device="cuda") for shape in self.shapes]
        torch.cuda.current_stream().synchronize()
        pointers = (ctypes.c_void_p * len(grads))(*[g.data_ptr() for g in grads])
        seconds = ctypes.c_double()
        call("ls200_sun_loss_backward", self.session.context, float(grad_output), pointers,
             len(grads), ctypes.byref(seconds))
        self.last_seconds["backward"] = float(seconds.value)
        return grads

    def checkpoints(self) -> dict:
        """Host copies of the last forward's checkpoints, sun directions and
        horizons (for the float64 reference and diagnostics)."""
        tiles = len(self.tiles)
        rays = tiles * PLANE * self.azimuth_count
        points = np.empty((rays, 4), dtype=np.float32)
        flags = np.empty(rays, dtype=np.uint8)
        directions = np.empty((tiles, self.time_count, PLANE, 2), dtype=np.float32)
        horizons = np.empty(rays, dtype=np.float32)
        call("ls200_sun_loss_checkpoints", self.session.context, points.ctypes.data,
             flags.ctypes.data, directions.ctypes.data, horizons.ctypes.data)
        shape = (tiles, PLANE, self.azimuth_count)
        return {"points": points.reshape(*shape, 4), "flags": flags.reshape(shape),
                "directions": directions, "horizons": horizons.reshape(shape)}

    # -- autograd -------------------------------------------------------------
    def loss(self, *heights):
        """Differentiable loss (a float64 scalar tensor) of the height tensors."""
        return _SunLoss.apply(self, *heights)


class StreamedSunLoss:
    """The loss of ``SunLossProblem`` over any number of tiles, evaluated in
    batches of ``batch_tiles``: each batch's forward pass is followed at once
    by its backward pass, so the argmax checkpoints of one batch only are
    resident (about 0.4 GB per tile at 1440 azimuths) however many tiles the
    loss covers.  The loss is a sum over tiles, so batch losses and
    gradients add up to the whole; ``loss`` returns it as an autograd scalar
    whose backward scales the gradient accumulated by the forward pass."""

    def __init__(self, session, dems: Sequence, tiles: Sequence[tuple[int, int]], weights,
                 sun_vectors, *, batch_tiles: int = 8, **options):
        if not 1 <= int(batch_tiles) <= 32:
            raise ValueError("batch_tiles must be between 1 and 32")
        self.tiles = [(int(tx), int(ty)) for tx, ty in tiles]
        if not self.tiles:
            raise ValueError("at least one tile")
        self.weights = np.asarray(weights, dtype=np.float32).reshape(len(self.tiles), PLANE)
        self.batch_tiles = int(batch_tiles)
        self.problem = SunLossProblem(session, dems, self.tiles[:self.batch_tiles],
                                      self.weights[:self.batch_tiles], sun_vectors, **options)
        self.last_seconds = {}

    def close(self) -> None:
        self.problem.close()

    def value_and_gradient(self, heights=None, grad_output: float = 1.0):
        """(loss, float64 gradients of grad_output x loss, one per DEM)."""
        import torch

        if heights is not None:
            self.problem.set_heights(heights)
        grads = [torch.zeros(shape, dtype=torch.float64, device="cuda")
                 for shape in self.problem.shapes]
        total = 0.0
        seconds = {"forward_march": 0.0, "forward_lighting": 0.0, "backward": 0.0}
        for start in range(0, len(self.tiles), self.batch_tiles):
            stop = start + self.batch_tiles
            self.problem.use_tiles(self.tiles[start:stop], self.weights[start:stop])
            total += self.problem.forward_value()
            for g, batch in zip(grads, self.problem.backward_value(grad_output)):
                g += batch
            for key in seconds:
                seconds[key] += self.problem.last_seconds[key]
        self.last_seconds = seconds
        return total, grads

    def loss(self, *heights):
        """Differentiable loss (a float64 scalar tensor) of the height tensors."""
        return _StreamedLoss.apply(self, *heights)


def psr_boundary_weights(psr, resolution_m: float, distance_m: float = 500.0) -> np.ndarray:
    """float32 weights, 1 on pixels within ``distance_m`` of the boundary of a
    PSR mask (pixels whose 4-neighbourhood holds both classes) and 0
    elsewhere: the region whose sun fraction the large sensitivity run
    differentiates.  Host preparation (scipy's Euclidean distance transform)."""
    from scipy import ndimage

    mask = np.asarray(psr) != 0
    boundary = np.zeros_like(mask)
    boundary[:-1, :] |= mask[:-1, :] != mask[1:, :]
    boundary[1:, :] |= mask[1:, :] != mask[:-1, :]
    boundary[:, :-1] |= mask[:, :-1] != mask[:, 1:]
    boundary[:, 1:] |= mask[:, 1:] != mask[:, :-1]
    if not boundary.any():
        return np.zeros(mask.shape, dtype=np.float32)
    distance = ndimage.distance_transform_edt(~boundary) * float(resolution_m)
    return (distance <= float(distance_m)).astype(np.float32)


def _function():
    import torch

    class SunLoss(torch.autograd.Function):
        @staticmethod
        def forward(ctx, problem, *heights):
            ctx.problem = problem
            ctx.dtypes = [h.dtype for h in heights]
            value = problem.forward_value(heights)
            return torch.tensor(value, dtype=torch.float64, device=heights[0].device)

        @staticmethod
        def backward(ctx, grad_output):
            grads = ctx.problem.backward_value(float(grad_output))
            return (None, *[g.to(dtype) for g, dtype in zip(grads, ctx.dtypes)])

    class StreamedLoss(torch.autograd.Function):
        @staticmethod
        def forward(ctx, streamed, *heights):
            ctx.dtypes = [h.dtype for h in heights]
            value, ctx.grads = streamed.value_and_gradient(heights)
            return torch.tensor(value, dtype=torch.float64, device=heights[0].device)

        @staticmethod
        def backward(ctx, grad_output):
            scale = grad_output.to(torch.float64)
            return (None, *[(scale * g).to(dtype) for g, dtype in zip(ctx.grads, ctx.dtypes)])

    return SunLoss, StreamedLoss


class _FunctionProxy:
    _classes = None

    def __init__(self, which: int):
        self.which = which

    def apply(self, *args):
        if _FunctionProxy._classes is None:
            _FunctionProxy._classes = _function()
        return _FunctionProxy._classes[self.which].apply(*args)


_SunLoss = _FunctionProxy(0)
_StreamedLoss = _FunctionProxy(1)
