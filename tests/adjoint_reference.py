"""Float64 PyTorch restatement of the differentiable sun-fraction loss, used
only by the tests to check the CUDA adjoint.

Given the forward's checkpoints (each ray's winning sample: position,
distance, pass, near flag) and sun directions, it recomputes the horizons
from DEM height tensors with torch operations (the reference's clamped
bilinear, near-field and spherical slope formulas), interpolates them at the
sun azimuth, applies the smooth disk fraction and sums the weighted means;
torch autograd then gives the gradient the adjoint kernels must match.
"""

from __future__ import annotations

import numpy as np
import torch

PLANE = 128 * 128


def _bilinear(heights: torch.Tensor, column: np.ndarray, row: np.ndarray):
    """The reference's clamped bilinear (clamp in float32 as the march does)."""
    height_px, width_px = heights.shape
    cmax = np.float32(width_px) - np.float32(1.0001)
    rmax = np.float32(height_px) - np.float32(1.0001)
    column = np.minimum(np.maximum(column.astype(np.float32), np.float32(0.0)), cmax)
    row = np.minimum(np.maximum(row.astype(np.float32), np.float32(0.0)), rmax)
    x0 = np.floor(column).astype(np.int64)
    y0 = np.floor(row).astype(np.int64)
    x1 = np.minimum(x0 + 1, width_px - 1)
    y1 = np.minimum(y0 + 1, height_px - 1)
    tx = torch.from_numpy(column.astype(np.float64) - x0)
    ty = torch.from_numpy(row.astype(np.float64) - y0)
    flat = heights.reshape(-1)

    def at(y, x):
        return flat[torch.from_numpy(y * width_px + x)]

    top = at(y0, x0) * (1 - tx) + at(y0, x1) * tx
    bottom = at(y1, x0) * (1 - tx) + at(y1, x1) * tx
    return top * (1 - ty) + bottom * ty


def reference_loss(heights, checkpoints: dict, tiles, weights, *, radius_deg: float,
                   observer_elevation_m: float, dem_radii, azimuth_count: int,
                   pin_to_device: bool = False):
    """Float64 loss of ``heights`` (float64 tensors, primary first).  With
    ``pin_to_device`` the horizon values are the device's (float32) and only
    their derivatives come from the float64 recomputation."""
    points = checkpoints["points"]          # [tiles, P, A, 4]
    flags = checkpoints["flags"]            # [tiles, P, A]
    directions = checkpoints["directions"]  # [tiles, T, P, 2]
    tile_count = len(tiles)
    weights = np.asarray(weights, dtype=np.float64).reshape(tile_count, PLANE)
    total = torch.zeros((), dtype=torch.float64)
    primary = heights[0]
    for t, (tx, ty) in enumerate(tiles):
        pixels = np.arange(PLANE)
        columns = tx + pixels % 128
        rows = ty + pixels // 128
        valid_pixel = (columns < primary.shape[1]) & (rows < primary.shape[0])
        observer = _bilinear(primary, np.where(valid_pixel, columns, 0).astype(np.float32),
                             np.where(valid_pixel, rows, 0).astype(np.float32))
        observer = observer + float(np.float32(observer_elevation_m))
        horizon = torch.full((PLANE, azimuth_count), -90.0, dtype=torch.float64)
        f = flags[t]
        for d, dem in enumerate(heights):
            mask = (f != 0xFF) & ((f >> 1) == d)
            if not mask.any():
                continue
            idx_p, idx_a = np.nonzero(mask)
            p = points[t][idx_p, idx_a]
            near = (f[idx_p, idx_a] & 1).astype(bool)
            h = _bilinear(dem, p[:, 0], p[:, 1])
            oz = observer[torch.from_numpy(idx_p)]
            dist = torch.from_numpy(p[:, 2].astype(np.float64))
            radius = float(np.float32(dem_radii[d]))
            rho = radius + oz
            z = ((radius + h) ** 2 - rho ** 2 - dist ** 2) / (2 * rho)
            lx2 = dist ** 2 - z ** 2
            far_slope = torch.where(lx2 > 0, z / torch.sqrt(torch.clamp(lx2, min=1e-30)),
                                    z / 1e-6)
            near_slope = (h - oz) / dist
            slope = torch.where(torch.from_numpy(near), near_slope, far_slope)
            degrees = torch.atan(slope) * (180.0 / np.pi)
            if pin_to_device:
                # Evaluate the lighting at the device's float32 horizons while
                # differentiating through the float64 recomputation.
                device = torch.from_numpy(
                    checkpoints["horizons"][t][idx_p, idx_a].astype(np.float64))
                degrees = degrees + (device - degrees).detach()
            horizon = horizon.index_put((torch.from_numpy(idx_p), torch.from_numpy(idx_a)),
                                        degrees)
        horizon = torch.clamp(horizon, min=-90.0)
        az = directions[t, :, :, 0].astype(np.float64)   # [T, P]
        el = torch.from_numpy(directions[t, :, :, 1].astype(np.float64))
        position = az * (azimuth_count / 360.0)
        left = position.astype(np.int64)
        fraction = torch.from_numpy(position - left)
        left = np.where(left >= azimuth_count, left - azimuth_count, left)
        right = np.where(left + 1 >= azimuth_count, 0, left + 1)
        pix = np.broadcast_to(pixels[None, :], left.shape)
        hl = horizon[torch.from_numpy(pix), torch.from_numpy(left)]
        hr = horizon[torch.from_numpy(pix), torch.from_numpy(right)]
        hz = hl + fraction * (hr - hl)
        u = (el - hz) / radius_deg
        inside = u.abs() < 1
        u_in = torch.where(inside, u, torch.zeros_like(u))
        inner = (torch.acos(-u_in) + u_in * torch.sqrt(1 - u_in * u_in)) / np.pi
        frac = torch.where(inside, inner, (u >= 1).to(torch.float64))
        w = torch.from_numpy(np.where(valid_pixel, weights[t], 0.0))
        total = total + (w * frac.mean(dim=0)).sum()
    return total
