"""Host logic of horizon generation: patch enumeration, tile naming and
completeness, the bounded pipeline (resume, progress, cancellation, error
propagation), the DEM container and pyramid cache, and the facade's
validation and error mapping (mirrors tests/test_horizon_api.py and
tests/numba_horizon/test_pipeline.py of the reference)."""

from __future__ import annotations

import threading
from pathlib import Path

import numpy as np
import pytest

import oracle
from lunarscout_b200 import horizon as horizon_module
from lunarscout_b200._native import CudaBackendError, CudaExecutionError
from lunarscout_b200.contract import DemGrid, ProjectionParameters
from lunarscout_b200.dem_io import (
    DemFormatError,
    load_dem,
    load_max_pyramid_cache,
    pyramid_cache_path,
    pyramid_layout,
    save_dem,
    write_max_pyramid_cache,
)
from lunarscout_b200.errors import (
    CudaError,
    HorizonGenerationError,
    InputError,
    OperationCancelledError,
)
from lunarscout_b200.file_format import RAW_FILE_BYTES, HorizonTileStore, normalize_tile
from lunarscout_b200.horizon import _HorizonProgressAdapter, generate_horizons
from lunarscout_b200.pipeline import (
    HorizonPipelineCancelled,
    HorizonProgress,
    enumerate_patches,
    run_bounded_pipeline,
)


def _dem(width=300, height=200) -> DemGrid:
    rng = np.random.default_rng(0)
    return DemGrid(rng.normal(0.0, 50.0, size=(height, width)).astype(np.float32),
                   np.array([-3000.0, 20.0, 0.0, 2000.0, 0.0, -20.0]),
                   ProjectionParameters.south_polar())


def _complete_bin(path: Path) -> Path:
    path.parent.mkdir(parents=True, exist_ok=True)
    with path.open("wb") as handle:
        handle.truncate(RAW_FILE_BYTES)
    return path


def _cbin_blocks(lengths) -> bytes:
    return b"".join(int(n).to_bytes(2, "little") + bytes(int(n)) for n in lengths)


# -- patches and the tile store ------------------------------------------------

def test_enumerate_patches_keeps_partial_edges_row_major():
    patches = enumerate_patches(300, 200)
    assert [(p.tile_x, p.tile_y, p.width, p.height) for p in patches] == [
        (0, 0, 128, 128), (128, 0, 128, 128), (256, 0, 44, 128),
        (0, 128, 128, 72), (128, 128, 128, 72), (256, 128, 44, 72)]
    assert [p.index for p in patches] == list(range(6))
    assert all(p.kernel_width == 128 and p.kernel_height == 128 for p in patches)
    with pytest.raises(ValueError):
        enumerate_patches(300, 200, include_partial_edges=False)
    for bad in ((0, 5), (5, -1), (True, 5), (5.0, 5)):
        with pytest.raises(ValueError):
            enumerate_patches(*bad)


def test_tile_names_and_lookup_precedence(tmp_path):
    store = HorizonTileStore(tmp_path)
    assert store.build_file_name(128, 256, 1.5, compress=True) == "horizon_00128_00256_015.cbin"
    assert store.build_file_name(0, 0, 0.0, compress=False) == "horizon_00000_00000_000.bin"
    assert store.build_path(128, 0, 0.0, compress=True) == \
        tmp_path / "00128" / "horizon_00128_00000_000.cbin"
    with pytest.raises(ValueError):
        store.build_file_name(0, 0, 100.0, compress=True)
    with pytest.raises(ValueError):
        store.build_file_name(100000, 0, 0.0, compress=True)
    names = [p.relative_to(tmp_path).as_posix() for p in store.candidate_paths(0, 128, 2.0)]
    assert names == ["00000/horizon_00000_00128_020.cbin", "00000/horizon_00000_00128_020.bin",
                     "horizon_00000_00128_020.cbin", "horizon_00000_00128_020.bin"]
    assert store.find_existing_path(0, 128, 2.0) is None
    legacy = _complete_bin(tmp_path / "horizon_00000_00128_020.bin")
    assert store.find_existing_path(0, 128, 2.0) == legacy
    assert HorizonTileStore(tmp_path, read_legacy_flat_files=False).find_existing_path(
        0, 128, 2.0) is None
    nested = _complete_bin(tmp_path / "00000" / "horizon_00000_00128_020.bin")
    assert store.find_existing_path(0, 128, 2.0) == nested


def test_structural_completeness(tmp_path):
    raw = _complete_bin(tmp_path / "a.bin")
    assert HorizonTileStore.is_complete(raw)
    with raw.open("ab") as handle:
        handle.write(bytes(28))                       # legacy metadata tail
    assert HorizonTileStore.is_complete(raw)
    with raw.open("ab") as handle:
        handle.write(bytes(1))
    assert not HorizonTileStore.is_complete(raw)
    good = tmp_path / "b.cbin"
    good.write_bytes(_cbin_blocks([2] * 16383 + [2880]))
    assert HorizonTileStore.is_complete(good)
    (tmp_path / "c.cbin").write_bytes(_cbin_blocks([2] * 16384) + b"\x00")
    assert not HorizonTileStore.is_complete(tmp_path / "c.cbin")
    (tmp_path / "d.cbin").write_bytes(_cbin_blocks([2] * 16383))
    assert not HorizonTileStore.is_complete(tmp_path / "d.cbin")
    (tmp_path / "e.cbin").write_bytes(_cbin_blocks([2] * 100 + [0] + [2] * 16283))
    assert not HorizonTileStore.is_complete(tmp_path / "e.cbin")
    (tmp_path / "f.cbin").write_bytes(_cbin_blocks([2] * 16383 + [2881]))
    assert not HorizonTileStore.is_complete(tmp_path / "f.cbin")
    assert not HorizonTileStore.is_complete(tmp_path / "missing.cbin")
    assert not HorizonTileStore.is_complete(tmp_path / "g.txt")


def test_normalize_pads_outside_the_valid_rectangle():
    valid = np.arange(3 * 2 * 1440, dtype=np.float32).reshape(6, 1440) % 40
    full = normalize_tile(valid, valid_width=2, valid_height=3).reshape(128, 128, 1440)
    np.testing.assert_array_equal(full[:3, :2].reshape(6, 1440), valid)
    assert np.all(full[3:] == -50.0) and np.all(full[:, 2:] == -50.0)
    with pytest.raises(ValueError):
        normalize_tile(np.full((6, 1440), np.nan, np.float32), valid_width=2, valid_height=3)
    with pytest.raises(ValueError):
        normalize_tile(valid, valid_width=0, valid_height=3)


def test_raw_write_is_staged_and_readable(tmp_path):
    store = HorizonTileStore(tmp_path)
    degrees = np.linspace(-10, 10, 16384 * 1440, dtype=np.float32).reshape(16384, 1440)
    path = store.write(0, 128, 0.5, degrees, compress=False)
    assert path.name == "horizon_00000_00128_005.bin" and store.is_complete(path)
    np.testing.assert_array_equal(store.read(0, 128, 0.5).reshape(16384, 1440), degrees)
    assert not list(tmp_path.rglob("*.tmp*"))


# -- the bounded pipeline --------------------------------------------------------

def _writer(store, compress=False):
    def write(patch, payload):
        return store.write_payload(patch.tile_y, patch.tile_x, 0.0, payload, compress=compress)
    return write


def test_pipeline_skips_complete_tiles_and_reports_progress(tmp_path):
    store = HorizonTileStore(tmp_path)
    patches = enumerate_patches(300, 200)
    _complete_bin(store.build_path(0, 128, 0.0, compress=False))
    (tmp_path / "00128").mkdir()
    store.build_path(128, 0, 0.0, compress=False).write_bytes(b"partial")   # incomplete
    computed, events = [], []

    def compute(patch):
        computed.append((patch.tile_x, patch.tile_y))
        return b"x" * 16

    result = run_bounded_pipeline(patches, store=store, compute_patch=compute,
                                  write_patch=_writer(store), progress_callback=events.append)
    assert result.skipped_patches == 1
    assert (128, 0) not in computed and (0, 128) in computed and len(computed) == 5
    assert len(result.output_paths) == 5
    assert [e.stage for e in events][:2] == ["prepare_patches", "process_patches"]
    assert events[-1].stage == "complete" and events[-1].processed_patches == 5
    done = [e.processed_patches for e in events if e.file_name]
    assert done == [1, 2, 3, 4, 5]
    assert result.maximum_writer_queue_depth <= 2


def test_pipeline_with_nothing_pending_reports_completion(tmp_path):
    store = HorizonTileStore(tmp_path)
    for patch in enumerate_patches(100, 100):
        _complete_bin(store.build_path(patch.tile_y, patch.tile_x, 0.0, compress=False))
    events = []
    result = run_bounded_pipeline(enumerate_patches(100, 100), store=store,
                                  compute_patch=lambda p: pytest.fail("nothing to compute"),
                                  write_patch=_writer(store), progress_callback=events.append)
    assert result.output_paths == () and result.skipped_patches == 1
    assert [e.stage for e in events] == ["prepare_patches", "complete"]


def test_pipeline_overwrite_recomputes(tmp_path):
    store = HorizonTileStore(tmp_path)
    _complete_bin(store.build_path(0, 0, 0.0, compress=False))
    result = run_bounded_pipeline(enumerate_patches(100, 100), store=store,
                                  compute_patch=lambda p: b"new", write_patch=_writer(store),
                                  skip_existing=False)
    assert result.skipped_patches == 0
    assert store.build_path(0, 0, 0.0, compress=False).read_bytes() == b"new"


def test_pipeline_cancellation_between_patches_keeps_published_tiles(tmp_path):
    store = HorizonTileStore(tmp_path)
    calls = {"n": 0}

    def compute(patch):
        calls["n"] += 1
        return b"t"

    written = []

    def write(patch, payload):
        path = _writer(store)(patch, payload)
        written.append(path)
        return path

    def cancelled():
        return len(written) >= 2

    with pytest.raises(HorizonPipelineCancelled):
        run_bounded_pipeline(enumerate_patches(600, 128), store=store, compute_patch=compute,
                             write_patch=write, cancellation_requested=cancelled)
    assert 2 <= len(written) < 5
    assert all(p.is_file() for p in written)
    assert not list(tmp_path.rglob("*.tmp*"))


def test_pipeline_propagates_the_first_compute_error(tmp_path):
    store = HorizonTileStore(tmp_path)

    def compute(patch):
        if patch.index == 2:
            raise CudaExecutionError("kernel failed")
        return b"ok"

    with pytest.raises(CudaExecutionError):
        run_bounded_pipeline(enumerate_patches(600, 128), store=store, compute_patch=compute,
                             write_patch=_writer(store))
    # Like the reference, tiles still queued when the error stops the
    # pipeline are dropped; nothing past the failing patch is published.
    assert len(list(tmp_path.rglob("*.bin"))) <= 2
    assert not list(tmp_path.rglob("*.tmp*"))


def test_pipeline_propagates_writer_errors_and_stops_computing(tmp_path):
    store = HorizonTileStore(tmp_path)
    computed = []
    gate = threading.Event()

    def compute(patch):
        computed.append(patch.index)
        if patch.index >= 1:
            gate.wait(timeout=5.0)
        return b"ok"

    def write(patch, payload):
        gate.set()
        raise OSError("disk full")

    with pytest.raises(OSError, match="disk full"):
        run_bounded_pipeline(enumerate_patches(128 * 20, 128), store=store,
                             compute_patch=compute, write_patch=write)
    assert len(computed) < 20


def test_pipeline_cancelled_before_start(tmp_path):
    with pytest.raises(HorizonPipelineCancelled):
        run_bounded_pipeline(enumerate_patches(100, 100), store=HorizonTileStore(tmp_path),
                             compute_patch=lambda p: b"", write_patch=lambda p, b: Path("x"),
                             cancellation_requested=lambda: True)


# -- DEM container and pyramid cache ----------------------------------------------

def test_dem_container_round_trip(tmp_path):
    dem = _dem()
    path = save_dem(tmp_path / "dem.npz", dem)
    loaded = load_dem(path)
    np.testing.assert_array_equal(loaded.elevation_m, dem.elevation_m)
    np.testing.assert_array_equal(loaded.geo_transform, dem.geo_transform)
    assert loaded.projection == dem.projection
    with pytest.raises(DemFormatError):
        load_dem(tmp_path / "dem.tif")
    (tmp_path / "bad.npz").write_bytes(b"not a zip")
    with pytest.raises(DemFormatError):
        load_dem(tmp_path / "bad.npz")


@pytest.mark.parametrize("shape", [(1, 1), (5, 3), (300, 200), (513, 1024)])
def test_pyramid_layout_matches_the_oracle(shape):
    width, height = shape
    levels, count = pyramid_layout(width, height)
    expected_levels, expected_count = oracle.pyramid_layout(width, height)
    np.testing.assert_array_equal(levels, expected_levels)
    assert count == expected_count


def test_pyramid_cache_round_trip_and_length_check(tmp_path):
    from lunarscout_b200.contract import PyramidArrays, map_parameters, projection_parameters

    dem = _dem()
    mips, levels = oracle.build_pyramid(dem.elevation_m)
    pyramid = PyramidArrays(dem.elevation_m, mips, levels, map_parameters(dem),
                            projection_parameters(dem))
    cache = pyramid_cache_path(tmp_path / "dem.npz")
    assert cache.name == "dem.pyr.bin"
    write_max_pyramid_cache(pyramid, cache)
    loaded = load_max_pyramid_cache(dem, cache)
    np.testing.assert_array_equal(loaded.mips, mips)
    np.testing.assert_array_equal(loaded.levels, levels)
    cache.write_bytes(cache.read_bytes()[:-4])
    with pytest.raises(ValueError):
        load_max_pyramid_cache(dem, cache)
    with pytest.raises(OSError):
        load_max_pyramid_cache(dem, tmp_path / "missing.pyr.bin")


# -- the public facade ---------------------------------------------------------------

@pytest.fixture
def dem_file(tmp_path):
    return save_dem(tmp_path / "dem.npz", _dem())


@pytest.mark.parametrize("paths, code", [
    ("dem.npz", "horizon_dem_paths_invalid"),
    ([], "horizon_dem_paths_empty"),
    ([None], "horizon_dem_paths_invalid"),
    (["missing.npz"], "horizon_dem_not_found"),
])
def test_facade_rejects_bad_dem_paths(tmp_path, paths, code):
    if isinstance(paths, list):
        paths = [tmp_path / p if isinstance(p, str) else p for p in paths]
    with pytest.raises(InputError) as info:
        generate_horizons(tmp_path / "out", paths)
    assert info.value.code == code


@pytest.mark.parametrize("options, code", [
    (dict(observer_height_m=100.0), "horizon_observer_height_invalid"),
    (dict(observer_height_m=-0.1), "horizon_observer_height_invalid"),
    (dict(observer_height_m=float("nan")), "horizon_observer_height_invalid"),
    (dict(observer_height_m=True), "horizon_observer_height_invalid"),
    (dict(compress=1), "horizon_option_invalid"),
    (dict(overwrite="no"), "horizon_option_invalid"),
    (dict(verbose=None), "horizon_option_invalid"),
    (dict(progress_callback=3), "horizon_callback_invalid"),
    (dict(cancellation_requested="x"), "horizon_callback_invalid"),
])
def test_facade_rejects_bad_options(tmp_path, dem_file, options, code):
    with pytest.raises(InputError) as info:
        generate_horizons(tmp_path / "out", [dem_file], **options)
    assert info.value.code == code


def test_facade_rejects_output_file_and_unreadable_dem(tmp_path, dem_file):
    target = tmp_path / "file"
    target.write_text("x")
    with pytest.raises(InputError) as info:
        generate_horizons(target, [dem_file])
    assert info.value.code == "horizon_output_is_file"
    other = tmp_path / "dem.tif"
    other.write_bytes(b"II*\x00")
    with pytest.raises(InputError) as info:
        generate_horizons(tmp_path / "out", [other])
    assert info.value.code == "horizon_dem_unreadable"


def test_facade_cancelled_before_work_touches_nothing(tmp_path, dem_file):
    with pytest.raises(OperationCancelledError) as info:
        generate_horizons(tmp_path / "out", [dem_file], cancellation_requested=lambda: True)
    assert info.value.code == "horizon_generation_cancelled"
    assert not (tmp_path / "out").exists()


@pytest.mark.parametrize("raised, kind, code", [
    (CudaBackendError("no device"), CudaError, "cuda_horizon_unavailable"),
    (CudaExecutionError("launch failed"), CudaError, "cuda_horizon_execution_failed"),
    (HorizonPipelineCancelled("stop"), OperationCancelledError, "horizon_generation_cancelled"),
    (OSError("disk full"), HorizonGenerationError, "horizon_storage_failed"),
    (RuntimeError("bad"), HorizonGenerationError, "horizon_generation_failed"),
])
def test_facade_maps_pipeline_failures(tmp_path, dem_file, monkeypatch, raised, kind, code):
    def fail(*args, **kwargs):
        raise raised

    monkeypatch.setattr(horizon_module, "run_horizon_pipeline", fail)
    with pytest.raises(kind) as info:
        generate_horizons(tmp_path / "out", [dem_file])
    assert info.value.code == code
    assert info.value.__cause__ is raised


def test_facade_without_a_device_raises_cuda_unavailable(tmp_path, dem_file):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(CudaError) as info:
        generate_horizons(tmp_path / "out", [dem_file])
    assert info.value.code == "cuda_horizon_unavailable"
    assert not list((tmp_path / "out").rglob("*.bin")) if (tmp_path / "out").exists() else True


def test_facade_callback_errors_propagate_unwrapped(tmp_path, dem_file, monkeypatch):
    class Boom(Exception):
        pass

    def fake_pipeline(dems, output, *, progress_callback, **kwargs):
        progress_callback(HorizonProgress(0, 1, 10.0, "prepare_patches", "go"))

    def explode(event):
        raise Boom()

    monkeypatch.setattr(horizon_module, "run_horizon_pipeline", fake_pipeline)
    with pytest.raises(Boom):
        generate_horizons(tmp_path / "out", [dem_file], progress_event_callback=explode)


def test_progress_adapter_fractions_are_monotonic_and_parse_tiles(tmp_path, capsys):
    fractions, events = [], []
    adapter = _HorizonProgressAdapter(tmp_path, verbose=True,
                                      progress_callback=fractions.append,
                                      progress_event_callback=events.append)
    adapter(HorizonProgress(0, 4, 10.0, "prepare_patches", "prep"))
    adapter(HorizonProgress(0, 4, 15.0, "process_patches", "start"))
    adapter(HorizonProgress(1, 4, 25.0, "process_patches", "one",
                            "horizon_00128_00256_000.cbin"))
    adapter(HorizonProgress(1, 4, 25.0, "process_patches", "again"))
    adapter(HorizonProgress(4, 4, 100.0, "complete", "done"))
    assert fractions == pytest.approx([0.1, 0.15, 0.15 + 0.85 / 4, 1.0])
    assert events[2].tile_y == 128 and events[2].tile_x == 256
    assert all(e.operation == "horizons" and e.backend == "cuda" for e in events)
    assert "horizons: using cuda backend" in capsys.readouterr().out


@pytest.mark.parametrize("options", [dict(batch_tiles=-1), dict(batch_tiles=True),
                                     dict(traversal="ladder"),
                                     dict(batch_tiles=4, traversal="fast")])
def test_grid_facade_rejects_bad_batch_options(tmp_path, options):
    from lunarscout_b200.horizon import generate_horizons_from_grids

    with pytest.raises(InputError) as info:
        generate_horizons_from_grids(tmp_path / "out", [_dem()], **options)
    assert info.value.code == "horizon_option_invalid"
