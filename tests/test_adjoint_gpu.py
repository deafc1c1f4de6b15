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
    assert abs(loss - float(ref)) <= 1e-6 * abs(loss)
    scale = np.abs(expected).max()
    assert scale > 0.0
    assert np.abs(grad - expected).max() <= 1e-5 * scale
    assert np.linalg.norm(grad - expected) <= 1e-6 * np.linalg.norm(expected)
    # The gradient reaches both the observers' own cells and distant terrain.
    assert np.count_nonzero(grad[160:224, 160:224]) > 3000
    assert np.count_nonzero(grad) > np.count_nonzero(grad[160:224, 160:224]) + 1000


def test_gradient_agrees_with_central_finite_differences(problem):
    p, dem, heights, _ = problem
    loss, grad = _forward_backward(p, heights)
    rng = np.random.default_rng(23)
    flat = np.abs(grad).ravel()
    strongest = np.argsort(flat)[-24:]
    nonzero = np.flatnonzero(flat > 1e-3 * flat.max())
    picks = np.unique(np.concatenate([strongest, rng.choice(nonzero, 16, replace=False)]))
    delta = 0.05
    errors = []
    for index in picks:
        y, x = divmod(int(index), dem.width)
        h = heights.clone()
        h[y, x] += delta
        plus = p.forward_value([h])
        h[y, x] -= 2 * delta
        minus = p.forward_value([h])
        fd = (plus - minus) / (2 * delta)
        errors.append(abs(fd - grad[y, x]) / max(abs(grad[y, x]), 1e-12))
    p.forward_value([heights])
    errors = np.array(errors)
    # The march's discrete choices can jump under a 5 cm change; the smooth
    # part must agree to 1e-3 for the large majority of cells.
    assert np.median(errors) <= 1e-3, errors
    assert np.mean(errors <= 1e-2) >= 0.8, errors


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
