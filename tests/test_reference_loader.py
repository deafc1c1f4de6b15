"""The loader of the reference installed under baseline/_ref (CPU): it
imports the reference's hot-path modules through a stub package, without
touching CUDA, and opens the reference's CUDA import gate only on request."""

from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "baseline"))
import load_reference  # noqa: E402

pytestmark = pytest.mark.skipif(not load_reference.available(),
                                reason="the reference is not installed under baseline/_ref")


def test_reference_modules_import_through_the_stub_package():
    nh = load_reference.import_reference()
    assert Path(nh.__file__).resolve().is_relative_to(load_reference.INSTALL.resolve())
    from lunarscout._numba_horizon import cuda_backend, generator, pipeline, psr

    assert callable(pipeline.run_bounded_pipeline)
    assert callable(generator.generate_patch_horizons)
    assert callable(psr.reduce_sun_vectors_for_psr)
    assert hasattr(cuda_backend, "CudaSession")


def test_reference_cpu_reduction_equals_the_oracle():
    """The installed reference and the oracle agree on the PSR vector
    reduction (the oracle is pinned to the same function by golden files)."""
    import numpy as np

    from oracle import products
    from lunarscout_b200 import synthetic

    load_reference.import_reference()
    from lunarscout._numba_horizon import geometry, psr

    ours = synthetic.config1_dem()
    dem = geometry.DemGrid(ours.elevation_m, np.array(ours.geo_transform),
                           geometry.ProjectionParameters.from_array(ours.projection.as_array()))
    sun = synthetic.sun_vectors(synthetic.hours_between("2030-01-01T00", "2030-03-01T00", 3.0))
    _, expected = psr.reduce_sun_vectors_for_psr(dem, sun)
    _, indices = products.reduce_sun_vectors(ours, sun)
    np.testing.assert_array_equal(indices, expected)


def test_numba_cuda_gate_is_opened_only_on_request():
    load_reference.import_reference()
    import lunarscout._cuda_runtime as runtime

    load_reference.import_reference(enable_numba_cuda=True)
    numba, cuda = runtime.import_numba_cuda()
    assert cuda.__name__ == "numba.cuda" and numba.__name__ == "numba"
