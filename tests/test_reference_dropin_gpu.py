"""The drop-in exercised through the reference's own code on the B200.

The reference lunarscout, installed unmodified under ``baseline/_ref`` and
imported through a stub package (its top-level package needs pyproj and
rasterio), runs its horizon pipeline exactly as ``ls/horizon.py:154-240``
wires it: the host Numba segment builder (``geometry.build_subpatch_segments_
numba``), ``generator.generate_patch_horizons``, ``HorizonBuffers.degrees``,
``pipeline.run_bounded_pipeline`` with its ``HorizonTileStore`` — with this
project's ``CudaSession`` swapped into ``cuda_backend`` the way
INTEGRATION.md's ``install()`` does it.  The reference's own Numba-CUDA
``CudaSession`` then runs the same patches on the same GPU: its tiles must
equal the ones written with the swapped session.

Skipped when the reference is not installed next to the repository.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "baseline"))
import load_reference  # noqa: E402

if not load_reference.available():  # pragma: no cover - depends on the install
    pytest.skip("the reference is not installed under baseline/_ref", allow_module_level=True)

OBSERVER_M = 1.5


@pytest.fixture(scope="module")
def reference():
    nh = load_reference.import_reference(enable_numba_cuda=True)
    from lunarscout._numba_horizon import (contract, cuda_backend, file_format, generator,
                                           geometry, pipeline)

    return dict(nh=nh, contract=contract, cuda_backend=cuda_backend, generator=generator,
                geometry=geometry, pipeline=pipeline, file_format=file_format)


@pytest.fixture(scope="module")
def plain_dems(reference):
    """The plain configuration's 512 x 512 DEM at 20 m (seed 1) as the
    reference's own DemGrid, and a 256 x 256 crop of it (4 tiles) for the
    pipeline runs."""
    from lunarscout_b200 import synthetic

    ours = synthetic.config1_dem()
    geometry = reference["geometry"]
    projection = geometry.ProjectionParameters.from_array(ours.projection.as_array())
    full = geometry.DemGrid(ours.elevation_m, np.array(ours.geo_transform, dtype=np.float64),
                            projection)
    shifted = np.array(ours.geo_transform, dtype=np.float64)
    shifted[0] += 128 * shifted[1]
    shifted[3] += 128 * shifted[5]
    crop = geometry.DemGrid(np.ascontiguousarray(ours.elevation_m[128:384, 128:384]), shifted,
                            projection)
    return full, crop


def _run_reference_pipeline(reference, dem, session_class, output, *, overwrite=False):
    """ls/horizon.py:154-240 for one DEM, with `session_class` as
    cuda_backend.CudaSession."""
    contract, geometry = reference["contract"], reference["geometry"]
    pipeline, file_format = reference["pipeline"], reference["file_format"]
    generator = reference["generator"]
    session = session_class(device_id=0, production_concurrency=1)
    pyramids = (session.build_max_pyramid(dem),)
    configuration = contract.ContractConfiguration(
        file_format.PATCH_SIZE, file_format.PATCH_SIZE, file_format.AZIMUTH_COUNT, 8, 1,
        dem.width, dem.height)

    def prepare(patch):
        values, _centers, _convergence = geometry.build_subpatch_segments_numba(
            [dem], tile_column=patch.tile_x, tile_row=patch.tile_y,
            tile_width=patch.kernel_width, azimuth_count=file_format.AZIMUTH_COUNT,
            maximum_distance_m=1_000_000.0, observer_elevation_m=OBSERVER_M, subpatch_size=8,
            grid_convergence=geometry.GridConvergenceInput(0.0, 0.0, 0.0), parallel=True)
        dem_ids = np.broadcast_to(np.arange(1, dtype=np.int32), values.shape[:-1]).copy()
        return contract.SegmentTensor(values, dem_ids, configuration)

    def processor_factory(_worker_id):
        def process(patch, segments):
            return generator.generate_patch_horizons(
                session, segments, pyramids, tile_column=patch.tile_x,
                tile_row=patch.tile_y, observer_elevation_m=OBSERVER_M).slopes
        return process

    def finalize(_patch, slopes):
        return contract.HorizonBuffers(slopes).degrees()

    try:
        return pipeline.run_bounded_pipeline(
            pipeline.enumerate_patches(dem.width, dem.height),
            store=file_format.HorizonTileStore(output), prepare_patch=prepare,
            processor_factory=processor_factory, finalize_patch=finalize,
            observer_elevation_m=OBSERVER_M, compress=True, skip_existing=not overwrite,
            prepared_queue_capacity=1, writer_queue_capacity=1, worker_count=1)
    finally:
        close = getattr(session, "close", None)
        if close is not None:
            close()


def test_reference_pipeline_runs_with_the_b200_session_and_resumes(reference, plain_dems,
                                                                  tmp_path):
    from lunarscout_b200.cuda_backend import CudaSession

    _, crop = plain_dems
    out = tmp_path / "swapped"
    result = _run_reference_pipeline(reference, crop, CudaSession, out)
    files = sorted(out.rglob("horizon_*.cbin"))
    assert len(files) == 4 and result.skipped_patches == 0
    first = {p.name: p.read_bytes() for p in files}
    # Resume: complete tiles are skipped; a removed tile is rewritten alone,
    # with the same bytes.
    again = _run_reference_pipeline(reference, crop, CudaSession, out)
    assert again.skipped_patches == 4
    files[1].unlink()
    resumed = _run_reference_pipeline(reference, crop, CudaSession, out)
    assert resumed.skipped_patches == 3
    assert {p.name: p.read_bytes() for p in sorted(out.rglob("horizon_*.cbin"))} == first
    # The reference's own reader decodes them back to 1440-azimuth degrees,
    # and its store finds them complete.
    tile = reference["file_format"].read_horizon_tile(files[0])
    assert tile.shape == (128 * 128, 1440) or tile.shape == (128, 128, 1440)
    assert all(reference["file_format"].HorizonTileStore.is_complete(p) for p in files)


def _reference_numba_session(reference):
    """The reference's own Numba-CUDA session, or a skip with the reason."""
    try:
        return reference["cuda_backend"].CudaSession(device_id=0)
    except Exception as error:  # the JIT or the device probe refused
        pytest.skip(f"reference Numba-CUDA unavailable on this GPU: {error!r}")


def test_reference_numba_cuda_tiles_equal_the_swapped_session_tiles(reference, plain_dems,
                                                                   tmp_path):
    from lunarscout_b200.cuda_backend import CudaSession

    _, crop = plain_dems
    _reference_numba_session(reference)
    ours = tmp_path / "b200"
    theirs = tmp_path / "numba"
    _run_reference_pipeline(reference, crop, CudaSession, ours)
    _run_reference_pipeline(reference, crop, reference["cuda_backend"].CudaSession, theirs)
    ours_files = {p.name: p.read_bytes() for p in ours.rglob("horizon_*.cbin")}
    theirs_files = {p.name: p.read_bytes() for p in theirs.rglob("horizon_*.cbin")}
    assert ours_files.keys() == theirs_files.keys() and len(ours_files) == 4
    assert ours_files == theirs_files


def test_reference_numba_cuda_march_matches_on_the_plain_tile(reference, plain_dems):
    """Slopes of one full 512 x 512 plain-configuration tile (1440 azimuths,
    1,000 km public range capped by the DEM) from the reference's Numba-CUDA
    kernel and from libls200, on the same host segments."""
    from lunarscout_b200.cuda_backend import CudaSession

    full, _ = plain_dems
    numba_session = _reference_numba_session(reference)
    geometry = reference["geometry"]
    values, _centers, _convergence = geometry.build_subpatch_segments_numba(
        [full], tile_column=192, tile_row=192, tile_width=128, azimuth_count=1440,
        maximum_distance_m=1_000_000.0, observer_elevation_m=OBSERVER_M, subpatch_size=8,
        grid_convergence=geometry.GridConvergenceInput(0.0, 0.0, 0.0), parallel=True)
    pyramid = numba_session.build_max_pyramid(full)
    kwargs = dict(tile_column=192, tile_row=192, tile_width=128, tile_height=128,
                  subpatch_size=8, observer_elevation_m=OBSERVER_M)
    theirs, _ = numba_session.subpatch_hierarchical_all_passes(values, [pyramid], **kwargs)
    session = CudaSession(0)
    try:
        ours, _ = session.subpatch_hierarchical_all_passes(values, [pyramid], **kwargs)
    finally:
        session.close()
    np.testing.assert_array_equal(ours, theirs)


def test_reference_pipeline_tiles_match_the_b200_generator(reference, plain_dems, tmp_path):
    """The same patches written by this project's own generator facade
    (``generate_horizons_from_grids``, device segment fitting) carry the same
    file names; the horizons differ only where the device FP64 segment fit
    and the reference's host Numba fit round a segment field differently
    (path error below 1e-5 px)."""
    from lunarscout_b200.contract import DemGrid, ProjectionParameters
    from lunarscout_b200.horizon import generate_horizons_from_grids
    from lunarscout_b200.cuda_backend import CudaSession

    _, crop = plain_dems
    swapped = tmp_path / "swapped"
    _run_reference_pipeline(reference, crop, CudaSession, swapped)
    from lunarscout_b200 import synthetic

    plain = synthetic.config1_dem()
    ours = DemGrid(crop.elevation_m, np.array(crop.geo_transform, dtype=np.float64),
                   ProjectionParameters.from_array(plain.projection.as_array()))
    generate_horizons_from_grids(tmp_path / "facade", [ours], observer_height_m=OBSERVER_M,
                                 compress=True)
    read = reference["file_format"].read_horizon_tile
    names = sorted(p.relative_to(swapped) for p in swapped.rglob("horizon_*.cbin"))
    assert names == sorted(p.relative_to(tmp_path / "facade")
                           for p in (tmp_path / "facade").rglob("horizon_*.cbin"))
    identical = 0
    for name in names:
        a = np.asarray(read(swapped / name), dtype=np.float64)
        b = np.asarray(read(tmp_path / "facade" / name), dtype=np.float64)
        assert a.shape == b.shape
        assert np.abs(a - b).max() <= 0.05
        identical += int((swapped / name).read_bytes() == (tmp_path / "facade" / name).read_bytes())
        assert np.mean(a == b) > 0.999
    print(f"byte-identical tiles: {identical} of {len(names)}")
