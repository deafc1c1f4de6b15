"""PSR-boundary weights of the large sensitivity run (host preparation)."""

from __future__ import annotations

import numpy as np

from lunarscout_b200.adjoint import psr_boundary_weights


def test_weights_cover_the_band_around_the_psr_boundary():
    y, x = np.mgrid[0:200, 0:200]
    psr = ((y - 100) ** 2 + (x - 100) ** 2 <= 40 ** 2).astype(np.uint8) * 255
    weights = psr_boundary_weights(psr, resolution_m=5.0, distance_m=50.0)
    assert weights.dtype == np.float32 and set(np.unique(weights)) == {0.0, 1.0}
    radius = np.hypot(y - 100, x - 100)
    assert np.all(weights[np.abs(radius - 40) <= 1.0] == 1.0)       # on the boundary
    assert np.all(weights[np.abs(radius - 40) >= 12.5] == 0.0)      # > 50 m away
    assert weights[100, 100 + 40 + 9] == 1.0 and weights[100, 100 - 40 - 12] == 0.0


def test_no_boundary_gives_zero_weights():
    assert not psr_boundary_weights(np.zeros((8, 8)), 5.0).any()
    assert not psr_boundary_weights(np.full((8, 8), 255), 5.0).any()
