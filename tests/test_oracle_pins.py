"""Pin the CPU oracle against the reference's golden captures (CPU only).

The fixtures come from the reference's own test data and from running the
reference's production kernel under Numba's CUDA simulator; see
tests/golden/make_golden.py.
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from oracle import segments as oseg
from conftest import load_golden

CAP = oracle.OPT_EXIT_CAP
PROD = oracle.PRODUCTION_MASK
CSHARP = oracle.CSHARP_MASK


def _interpolated(segments4, shifts=((4, 4), (-4, 4), (4, -4), (-4, -4))):
    """The reference tests' centre-of-four interpolation (tx = ty = 0.5)."""
    s = np.array(segments4, dtype=np.float32, copy=True)
    d = np.asarray(shifts, dtype=np.float32)
    s[:, 0] += d[:, 0]
    s[:, 2] += d[:, 0]
    s[:, 1] += d[:, 1]
    s[:, 3] += d[:, 1]
    half = np.float32(0.5)
    top = s[0] + (s[1] - s[0]) * half
    bottom = s[2] + (s[3] - s[2]) * half
    seg = (top + (bottom - top) * half).astype(np.float32)
    return seg[list(oracle.SEGMENT_MARCH_FIELDS)]


def _same(a, b):
    return np.array_equal(np.nan_to_num(a, nan=-12345.0), np.nan_to_num(b, nan=-12345.0))


def _passes(arrays, pyramids, mask, precision="f32"):
    out = []
    for p in range(2):
        slopes, _ = oracle.march_pass(
            arrays["segments"], pyramids[0], pyramids[p], tile_column=20, tile_row=20,
            tile_width=1, tile_height=1, subpatch_size=8, pass_index=p, mask=mask,
            precision=precision)
        out.append(slopes[0])
    return np.array(out)


def test_oracle_reproduces_the_csharp_traversal_trace_exactly(production_case):
    arrays, pyramids = production_case
    seg = _interpolated(arrays["csharp_trace_segments"])
    value, trace = oracle.hierarchy_maximum(
        seg, pyramids[1], observer_z=float(arrays["csharp_trace_observer_z"]),
        radius=1737400.0, resolution=30.0, pass_index=1, mask=CSHARP | CAP, capacity=4096)
    expected = arrays["csharp_trace"]
    assert trace.shape == expected.shape == (932, 12)
    assert _same(trace, expected)
    assert np.float32(value) == arrays["csharp_trace_maximum_slope"]


def test_oracle_reproduces_the_csharp_bilinear_boundary_trace(production_case):
    arrays, _ = production_case
    from lunarscout_b200.contract import PyramidArrays

    elevation = np.ascontiguousarray(arrays["boundary_elevation"], dtype=np.float32)
    mips, levels = oracle.build_pyramid(elevation)
    pyramid = PyramidArrays(elevation, mips, levels, np.zeros(11, np.float32),
                            np.zeros(6, np.float32))
    seg = _interpolated(arrays["boundary_segments"])
    value, trace = oracle.hierarchy_maximum(
        seg, pyramid, observer_z=float(arrays["boundary_observer_z"]),
        radius=float(arrays["boundary_radius"]), resolution=float(arrays["boundary_resolution"]),
        pass_index=0, mask=CSHARP | CAP, capacity=4096)
    expected = arrays["boundary_trace"]
    assert trace.shape == expected.shape
    # Structure and decisions exactly; values to the JSON's printed precision.
    np.testing.assert_array_equal(trace[:, [2, 3, 4, 11]], expected[:, [2, 3, 4, 11]])
    np.testing.assert_allclose(trace, expected, rtol=0, atol=1e-9, equal_nan=True)
    assert abs(value - float(arrays["boundary_maximum_slope"])) < 1e-7


def test_oracle_with_the_superseded_cell_exit_cap_matches_csharp_per_dem_slopes(production_case):
    arrays, pyramids = production_case
    got = _passes(arrays, pyramids, CSHARP | CAP)
    expected = arrays["csharp_per_dem_slopes"]
    np.testing.assert_allclose(got, expected, rtol=0, atol=3e-10)


def test_current_production_march_differs_from_the_older_capture_only_at_the_cap(production_case):
    """The reference removed the level-0 cell-exit cap after this capture
    (CHANGELOG 'Removed the level-0 cell-exit cap'); only the 1-pixel
    obstacle ray at azimuth 360 of the outer DEM pass depends on it."""
    arrays, pyramids = production_case
    got = _passes(arrays, pyramids, PROD)
    expected = arrays["csharp_per_dem_slopes"]
    bad = np.argwhere(np.abs(got - expected) > 3e-7)
    assert bad.tolist() == [[1, 360]]


def test_oracle_matches_the_reference_production_kernel_run_by_the_simulator(production_case):
    """The simulator executes the reference kernel with NumPy float32 ops and
    no contraction: the oracle with no fused multiply-adds is bit-identical."""
    arrays, pyramids = production_case
    got = _passes(arrays, pyramids, 0)
    np.testing.assert_array_equal(got[0], arrays["reference_sim_pass0"])
    np.testing.assert_array_equal(np.maximum(got[0], got[1]), arrays["reference_sim_final"])
    # The production (fused) arithmetic stays within the reference's 3e-7
    # slope tolerance of the unfused simulation.
    fused = _passes(arrays, pyramids, PROD)
    np.testing.assert_allclose(np.maximum(fused[0], fused[1]), arrays["reference_sim_final"],
                               rtol=0, atol=3e-7)


def test_fp64_restatement_agrees_with_fp32_march_within_the_horizon_gate(production_case):
    arrays, pyramids = production_case
    f32 = _passes(arrays, pyramids, PROD)
    f64 = _passes(arrays, pyramids, PROD, precision="f64")
    finite = np.isfinite(f32) & np.isfinite(f64)
    assert np.array_equal(np.isfinite(f32), np.isfinite(f64))
    error_deg = np.abs(np.degrees(np.arctan(f32[finite].astype(np.float64)))
                       - np.degrees(np.arctan(f64[finite])))
    assert error_deg.max() <= 0.01


def test_oracle_pyramids_match_every_csharp_capture():
    arrays = load_golden("pyramids.npz")
    names = [str(n) for n in arrays["names"]]
    assert names
    for index in range(len(names)):
        levels = arrays[f"p{index}_levels"]
        level0 = arrays[f"p{index}_level0"]
        mips, got_levels = oracle.build_pyramid(level0)
        np.testing.assert_array_equal(got_levels, levels)
        for level in range(1, len(levels)):
            _, offset, width, height = levels[level]
            np.testing.assert_array_equal(
                mips[offset:offset + width * height].reshape(height, width),
                arrays[f"p{index}_level{level}"])


def test_oracle_pyramid_invalid_value_rules():
    arrays = load_golden("pyramids.npz")
    source = arrays["invalid_elevation"]
    assert np.isnan(source).sum() == 1 and np.isposinf(source).sum() == 1
    mips, levels = oracle.build_pyramid(source)
    np.testing.assert_array_equal(levels, arrays["invalid_levels"])
    np.testing.assert_array_equal(mips[:4].reshape(2, 2), arrays["invalid_level1"])
    np.testing.assert_array_equal(mips[4:5].reshape(1, 1), arrays["invalid_level2"])


def _path_error(a, b):
    a = a.reshape(-1, 18).astype(np.float64)
    b = b.reshape(-1, 18).astype(np.float64)
    lo = np.maximum(a[:, 12], b[:, 12])
    hi = np.minimum(a[:, 13], b[:, 13])
    t = np.linspace(0.0, 1.0, 65)[None, :]
    d = lo[:, None] + (hi - lo)[:, None] * t

    def evaluate(s):
        dd = d - s[:, 12:13]
        x = s[:, 0:1] + sum(s[:, 3 + k:4 + k] * dd ** k for k in range(1, 5))
        y = s[:, 1:2] + sum(s[:, 7 + k:8 + k] * dd ** k for k in range(1, 5))
        return x, y

    ax, ay = evaluate(a)
    bx, by = evaluate(b)
    return float(np.max(np.hypot(ax - bx, ay - by)))


class _Dem:
    def __init__(self, elevation, transform, projection):
        from lunarscout_b200.contract import ProjectionParameters

        self.elevation_m = np.ascontiguousarray(elevation, dtype=np.float32)
        self.geo_transform = np.ascontiguousarray(transform, dtype=np.float64)
        self.projection = ProjectionParameters.from_array(projection)


def halo_dems(arrays):
    return [_Dem(arrays[f"dem{i}_elevation"], arrays[f"dem{i}_geo_transform"],
                 arrays[f"dem{i}_projection"]) for i in range(2)]


def test_oracle_segments_match_reference_numba_and_csharp():
    arrays = load_golden("segments_halo.npz")
    tc, tr, tw, _th, sub, az, dist = (int(v) for v in arrays["config"])
    got = oseg.build_segments(halo_dems(arrays), tile_column=tc, tile_row=tr, tile_width=tw,
                              azimuth_count=az, maximum_distance_m=float(dist),
                              observer_elevation_m=0.0, subpatch_size=sub)
    reference = arrays["reference_numba_segments"]
    assert got.shape == reference.shape
    # Same fields exactly except quartic coefficients of an ill-conditioned
    # fit, whose paths agree to well below a micro-pixel.
    assert _path_error(got, reference) < 1e-7
    np.testing.assert_array_equal(got[..., 12:15], reference[..., 12:15])
    # The reference's own C# tolerance (test_phase3_geometry.py:225).
    assert _path_error(got, arrays["csharp_segments"]) < 1e-5
    np.testing.assert_allclose(got, arrays["csharp_segments"], rtol=0, atol=1e-5)


def _numba_case():
    from lunarscout_b200 import synthetic
    from lunarscout_b200.contract import PyramidArrays, map_parameters, projection_parameters

    arrays = load_golden("numba_cuda_b200.npz")
    pyramids = []
    for dem in (synthetic.config1_dem(), synthetic.regional_dem()):
        mips, levels = oracle.build_pyramid(dem.elevation_m)
        pyramids.append(PyramidArrays(dem.elevation_m, mips, levels, map_parameters(dem),
                                      projection_parameters(dem)))
    column, row = (int(v) for v in arrays["tile"])
    common = dict(tile_column=column, tile_row=row,
                  observer_elevation_m=float(arrays["observer_elevation_m"]))
    return arrays, pyramids, common


def test_oracle_reproduces_the_reference_numba_cuda_march_on_the_b200():
    """The reference's own Numba-CUDA kernel, run on a B200 (two DEM passes,
    16,384 pixels x 12 azimuths): the production mask reproduces every slope
    bit for bit; the C# captures' mask (local_x^2 fused on dist * dist) does
    not."""
    arrays, pyramids, common = _numba_case()
    got, _ = oracle.march_all_passes(arrays["segments"], pyramids, **common)
    np.testing.assert_array_equal(got, arrays["slopes"])
    csharp, _ = oracle.march_all_passes(arrays["segments"], pyramids, mask=CSHARP, **common)
    assert np.count_nonzero(csharp != arrays["slopes"]) > 0
    assert np.isfinite(got).mean() > 0.99
