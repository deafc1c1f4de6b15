"""The DEM adjoint of the time-integrated sun fraction on the B200: the loss
and its gradient against a float64 PyTorch autograd restatement (64 x 64
weighted sub-tile, 360 azimuths), central finite differences at +-0.05 m,
and repeatability."""

from __future__ import annotations

import numpy as np
import pytest

from adjoint_reference import reference_loss

pytestmark = pytest.mark.gpu

AZ = 360
OBSERVER = 1.5


@pytest.fixture(scope="module")
def problem(cuda_session):
    import torch

    from lunarscout_b200.adjoint import SunLossProblem
    from lunarscout_b200.synthetic import SyntheticDemSpec, hours_between, sun_vectors, \
        synthetic_dem

    dem = synthetic_dem(SyntheticDemSpec(384, 10.0, craters=25, crater_max_m=1500.0, seed=21))
    weights = np.zeros((128, 128), dtype=np.float32)
    rng = np.random.default_rng(22)
    weights[32:96, 32:96] = rng.uniform(0.0, 1.0, size=(64, 64))
    vectors = sun_vectors(hours_between("2030-03-01T00", "2030-03-05T00", 2.0))
    p = SunLossProblem(cuda_session, [dem], [(128, 128)], weights[None], vectors,
                       maximum_distance_m=20_000.0, observer_elevation_m=OBSERVER,
                       azimuth_count=AZ, traversal="ladder")
    heights = torch.from_numpy(dem.elevation_m).cuda()
    yield p, dem, heights, weights
    p.close()


def _forward_backward(p, heights):
    loss = p.forward_value([heights])
    (grad,) = p.backward_value(1.0)
    return loss, grad.cpu().numpy()


def test_loss_and_gradient_match_the_float64_autograd_reference(problem):
    import torch

    p, dem, heights, weights = problem
    loss, grad = _forward_backward(p, heights)
    chk = p.checkpoints()
    h64 = torch.from_numpy(dem.elevation_m.astype(np.float64)).requires_grad_(True)
    ref = reference_loss([h64], chk, [(128, 128)], weights[None],
                         radius_deg=p.disk_radius_deg, observer_elevation_m=OBSERVER,
                         dem_radii=[dem.projection.radius_m], azimuth_count=AZ)
    ref.backward()
    expected = h64.grad.numpy()
    assert loss > 0.0
    # float32 horizons on the device, float64 recomputed here: u = (el - h)/r
    # amplifies a horizon's last-bit rounding by 1/r.
    assert abs(loss - float(ref.detach())) <= 2e-5 * abs(loss)
    scale = np.abs(expected).max()
    assert scale > 0.0
    # Unpinned, the sun-disk slope dF/du (infinite at |u| = 1) sees the
    # float32 / float64 horizon difference: agreement to 1e-3 of the scale.
    assert np.abs(grad - expected).max() <= 1e-3 * scale
    # Pinned to the device's horizon values, only the adjoint's own
    # arithmetic differs (it takes d degrees / d slope at the float32 slope
    # of the checkpoint): agreement to 1e-6.
    h64 = torch.from_numpy(dem.elevation_m.astype(np.float64)).requires_grad_(True)
    pinned = reference_loss([h64], chk, [(128, 128)], weights[None],
                            radius_deg=p.disk_radius_deg, observer_elevation_m=OBSERVER,
                            dem_radii=[dem.projection.radius_m], azimuth_count=AZ,
                            pin_to_device=True)
    pinned.backward()
    exact = h64.grad.numpy()
    assert np.abs(grad - exact).max() <= 1e-6 * scale
    assert np.linalg.norm(grad - exact) <= 1e-6 * np.linalg.norm(exact)
    # The gradient reaches both the observers' own cells and the terrain that
    # casts their horizons (only where the sun disk straddles a horizon).
    assert np.count_nonzero(grad[160:224, 160:224]) > 500
    assert np.count_nonzero(grad) > np.count_nonzero(grad[160:224, 160:224]) + 100


def _finite_difference_picks(grad, count_strong=24, count_random=16, seed=23):
    rng = np.random.default_rng(seed)
    flat = np.abs(grad).ravel()
    strongest = np.argsort(flat)[-count_strong:]
    nonzero = np.flatnonzero(flat > 1e-3 * flat.max())
    return np.unique(np.concatenate([strongest,
                                     rng.choice(nonzero, count_random, replace=False)]))


OBSERVERS = (slice(160, 224), slice(160, 224))  # the weighted pixels' own cells


def _replay_fd_errors(p, dem, heights, grad, cells, delta):
    errors = []
    for index in cells:
        y, x = divmod(int(index), dem.width)
        h = heights.clone()
        h[y, x] += delta
        plus = p.replay_value([h])
        h[y, x] -= 2 * delta
        minus = p.replay_value([h])
        fd = (plus - minus) / (2 * delta)
        errors.append(abs(fd - grad[y, x]) / abs(grad[y, x]))
    p.set_heights([heights])
    return np.array(errors)


def test_gradient_agrees_with_central_finite_differences(problem):
    """Central differences of the loss with the march's sampling held fixed
    (the function the adjoint differentiates).  Terrain cells move samples of
    other pixels' rays: +-0.05 m agrees to 1e-3.  An observer's own cell
    shifts all of its rays at once, and +-0.05 m moves near-field horizons by
    a sizeable part of the disk radius, where the loss is curved; there the
    step is 2^-9 m (exact in float32 heights)."""
    p, dem, heights, _ = problem
    p.forward_value([heights])
    p.replay_value()
    (grad,) = p.backward_value(1.0)
    grad = grad.cpu().numpy()
    observer = np.zeros_like(grad, dtype=bool)
    observer[OBSERVERS] = True
    magnitude = np.abs(grad)
    rng = np.random.default_rng(23)
    terrain = np.flatnonzero((~observer).ravel() & (magnitude.ravel() > 1e-3 * magnitude.max()))
    own = np.flatnonzero(observer.ravel() & (magnitude.ravel() > 1e-3 * magnitude.max()))
    terrain_errors = _replay_fd_errors(p, dem, heights, grad,
                                       rng.choice(terrain, min(24, terrain.size), replace=False),
                                       0.05)
    own_errors = _replay_fd_errors(p, dem, heights, grad,
                                   rng.choice(own, min(24, own.size), replace=False), 2.0 ** -9)
    # Terrain next to the observers carries near-field samples too, so a few
    # cells show the same curvature at 0.05 m.
    assert np.median(terrain_errors) <= 1e-4, terrain_errors
    assert np.mean(terrain_errors <= 1e-3) >= 0.9, terrain_errors
    assert terrain_errors.max() <= 1e-2, terrain_errors
    assert np.median(own_errors) <= 2e-3, own_errors
    assert np.mean(own_errors <= 1e-2) >= 0.8, own_errors


def _central_difference(p, heights, y, x, step):
    """Central difference of the replayed loss at cell (y, x), divided by the
    float32 heights' actual separation (a step the heights cannot hold
    exactly would otherwise bias the quotient)."""
    h = heights.clone()
    base = float(heights[y, x])
    h[y, x] = base + step
    upper = float(h[y, x])
    plus = p.replay_value([h])
    h[y, x] = base - step
    lower = float(h[y, x])
    minus = p.replay_value([h])
    return (plus - minus) / (upper - lower)


STEPS = (2.0 ** -4, 2.0 ** -6, 2.0 ** -8, 2.0 ** -10, 2.0 ** -12)


def _sweep(p, heights, grad, cells, steps=STEPS):
    """Relative error of the central difference at every step of `steps` and
    of the Richardson extrapolation of the two smallest (steps a factor 4
    apart: (16 D(s / 4) - D(s)) / 15 cancels the s^2 term)."""
    raw = np.zeros((len(cells), len(steps)))
    extrapolated = np.zeros(len(cells))
    for i, index in enumerate(cells):
        y, x = divmod(int(index), grad.shape[1])
        d = [_central_difference(p, heights, y, x, step) for step in steps]
        raw[i] = [abs(v - grad[y, x]) / abs(grad[y, x]) for v in d]
        extrapolated[i] = abs((16.0 * d[-1] - d[-2]) / 15.0 - grad[y, x]) / abs(grad[y, x])
    p.set_heights([heights])
    return raw, extrapolated


def test_observer_cell_differences_converge_to_the_gradient(problem):
    """An observer's own cell moves every one of its rays at once, and a
    near-field sample 1 m away turns a height change of s metres into an
    elevation change of about s radians: at +-0.05 m that is ~3 deg, ten disk
    radii, so the loss is far from linear over the step.  Shrinking the step
    shows the central differences converging to the adjoint (error ~ s^2),
    and the Richardson extrapolation of the two smallest steps agrees to
    1e-3 in the median, on the observer cells with the largest gradients and
    on 200 random cells with a gradient (observers and terrain)."""
    p, dem, heights, _ = problem
    p.forward_value([heights])
    p.replay_value()
    (grad,) = p.backward_value(1.0)
    grad = grad.cpu().numpy()
    magnitude = np.abs(grad)
    live = magnitude > 1e-3 * magnitude.max()
    observer = np.zeros_like(live)
    observer[OBSERVERS] = True
    own = np.flatnonzero((observer & live).ravel())
    strongest_own = own[np.argsort(magnitude.ravel()[own])[-24:]]
    raw, extrapolated = _sweep(p, heights, grad, strongest_own)
    medians = np.median(raw, axis=0)
    assert medians[-1] < medians[0] / 20.0, medians          # converging with the step
    assert np.median(extrapolated) <= 1e-3, (medians, extrapolated)
    rng = np.random.default_rng(25)
    random_cells = rng.choice(np.flatnonzero(live.ravel()), 200, replace=False)
    _, extrapolated = _sweep(p, heights, grad, random_cells, STEPS[-2:])
    assert np.median(extrapolated) <= 1e-3, np.median(extrapolated)
    assert np.mean(extrapolated <= 1e-2) >= 0.9, np.mean(extrapolated <= 1e-2)


def test_full_march_finite_differences_are_reported(problem):
    """Through the full march a 5 cm change also moves step positions and can
    switch the winning sample; those differences are measured, not gated
    beyond a sign check."""
    p, dem, heights, _ = problem
    loss, grad = _forward_backward(p, heights)
    same_sign = []
    for index in _finite_difference_picks(grad, 12, 8, seed=24):
        y, x = divmod(int(index), dem.width)
        h = heights.clone()
        h[y, x] += 0.05
        plus = p.forward_value([h])
        h[y, x] -= 0.1
        minus = p.forward_value([h])
        same_sign.append(np.sign(plus - minus) == np.sign(grad[y, x]))
    p.forward_value([heights])
    assert np.mean(same_sign) >= 0.7


def test_repeated_calls_are_consistent_and_autograd_wraps_them(problem):
    import torch

    p, dem, heights, _ = problem
    loss_a, grad_a = _forward_backward(p, heights)
    loss_b, grad_b = _forward_backward(p, heights)
    assert loss_a == loss_b
    np.testing.assert_allclose(grad_a, grad_b, rtol=1e-12, atol=1e-18)
    h = heights.clone().requires_grad_(True)
    loss = p.loss(h)
    loss.backward()
    assert loss.dtype == torch.float64 and float(loss) == loss_a
    np.testing.assert_allclose(h.grad.cpu().numpy(), grad_a.astype(np.float32), rtol=1e-6,
                               atol=1e-12)
    assert p.last_seconds["backward"] > 0.0


def test_adjoint_rejects_inconsistent_problems(problem, cuda_session):
    import torch

    from lunarscout_b200.adjoint import SunLossProblem

    p, dem, heights, weights = problem
    with pytest.raises(ValueError):
        p.set_heights([heights[:10]])
    with pytest.raises(ValueError):
        SunLossProblem(cuda_session, [dem], [(0, 0)], np.zeros(5), np.ones((3, 3)))
    with pytest.raises(ValueError):
        p.backward_value.__self__.set_heights([heights, heights])
    assert torch.isfinite(heights).all()


def test_streamed_batches_add_up_to_the_one_shot_loss_and_gradient(cuda_session):
    import torch

    from lunarscout_b200.adjoint import StreamedSunLoss, SunLossProblem
    from lunarscout_b200.synthetic import SyntheticDemSpec, hours_between, sun_vectors, \
        synthetic_dem

    dem = synthetic_dem(SyntheticDemSpec(512, 10.0, craters=30, crater_max_m=1500.0, seed=23))
    tiles = [(128, 128), (256, 128), (128, 256), (256, 256), (384, 384)]
    weights = np.random.default_rng(24).uniform(0.0, 1.0, (len(tiles), 128, 128))
    vectors = sun_vectors(hours_between("2030-03-01T00", "2030-03-03T00", 4.0))
    options = dict(maximum_distance_m=5_000.0, observer_elevation_m=OBSERVER, azimuth_count=AZ)
    heights = torch.from_numpy(dem.elevation_m).cuda()
    whole = SunLossProblem(cuda_session, [dem], tiles, weights, vectors, **options)
    streamed = StreamedSunLoss(cuda_session, [dem], tiles, weights, vectors, batch_tiles=2,
                               **options)
    try:
        loss = whole.forward_value([heights])
        (grad,) = whole.backward_value(1.0)
        value, (streamed_grad,) = streamed.value_and_gradient([heights])
        assert loss > 0.0
        assert abs(value - loss) <= 1e-12 * abs(loss)
        grad, streamed_grad = grad.cpu().numpy(), streamed_grad.cpu().numpy()
        scale = np.abs(grad).max()
        assert scale > 0.0
        assert np.abs(streamed_grad - grad).max() <= 1e-12 * scale
        h = heights.clone().requires_grad_(True)
        out = streamed.loss(h)
        (2.5 * out).backward()
        assert abs(float(out) - value) <= 1e-12 * abs(value)
        np.testing.assert_allclose(h.grad.cpu().numpy(), (2.5 * streamed_grad).astype(np.float32),
                                   rtol=1e-6, atol=1e-6 * 2.5 * scale)
    finally:
        whole.close()
        streamed.close()
