"""The safe-haven oracle and month-band helpers against the reference's own
outputs (tests/golden/safe_haven_reference.npz, made by make_golden.py from
safe_haven.py), and the device reducer's run-end crediting against the
oracle's per-step crediting on random streams (CPU, no device)."""

from __future__ import annotations

from datetime import datetime

import numpy as np
import pytest

from oracle import products
from conftest import load_golden

from lunarscout_b200.safe_haven import month_bands, month_indices


@pytest.fixture(scope="module")
def golden():
    return load_golden("safe_haven_reference.npz")


def _bands(flat):
    values = [datetime.fromisoformat(str(v)) for v in flat]
    return tuple(zip(values[0::2], values[1::2]))


def test_oracle_matches_reference_on_reference_lighting_streams(golden):
    lighting = load_golden("lighting_reference.npz")
    bands = _bands(golden["a_bands"])
    got = products.safe_haven(lighting["fractions"], lighting["margins"], golden["a_months"],
                              len(bands), sunlight_threshold=float(golden["a_sunlight"]),
                              earth_threshold_deg=float(golden["a_earth"]), time_step_hours=6.0)
    np.testing.assert_array_equal(got, golden["a_out"])
    assert np.isfinite(got).any() and np.isnan(got).any()


@pytest.mark.parametrize("case,hours", [("b", 6.0), ("c", 1.5)])
def test_oracle_matches_reference_on_synthetic_streams(golden, case, hours):
    months = golden[f"{case}_months"]
    band_count = golden[f"{case}_out"].shape[0]
    got = products.safe_haven(golden["b_fractions"], golden["b_margins"], months, band_count,
                              sunlight_threshold=0.2, earth_threshold_deg=2.0,
                              time_step_hours=hours)
    np.testing.assert_array_equal(got, golden[f"{case}_out"])
    assert np.isnan(got[:, 0, :3]).all() and np.isnan(got[:, 1, :3]).all()
    assert (got[np.isfinite(got)] > 0).any()


def test_month_bands_and_indices_match_reference(golden):
    times = [datetime.fromisoformat(str(v)) for v in golden["b_times"]]
    bands = month_bands(times)
    assert bands == _bands(golden["b_bands"])
    np.testing.assert_array_equal(month_indices(times, bands), golden["b_months"])
    shuffled = [datetime.fromisoformat(str(v)) for v in golden["c_times"]]
    np.testing.assert_array_equal(month_indices(shuffled, bands[1:]), golden["c_months"])
    assert (golden["c_months"] == -1).any()
    strings = [t.isoformat().replace("+00:00", "Z") for t in times]
    assert month_bands(strings) == bands
    assert month_bands([]) == ()


def test_month_bands_cross_the_year():
    bands = month_bands(["2029-12-31T23:00Z", "2030-01-01T00:00Z"])
    assert [(a.month, b.month, b.year) for a, b in bands] == [(12, 1, 2030), (1, 2, 2030)]


def _run_end_crediting(low, outage, months, band_count, hours):
    """The device reducer's algorithm (lighting.cu haven_kernel) in Python:
    credit a run once, at its end, to the bands it touched."""
    count, height, width = low.shape
    out = np.empty((band_count, height, width), dtype=np.float32)
    for y in range(height):
        for x in range(width):
            longest = np.zeros(band_count, dtype=np.int64)
            flags = np.zeros(band_count, dtype=np.int64)
            run, touched = 0, set()
            for t in range(count):
                if low[t, y, x]:
                    run += 1
                else:
                    for b in touched:
                        longest[b] = max(longest[b], run)
                    touched, run = set(), 0
                m = int(months[t])
                if m >= 0:
                    flags[m] |= 1 if outage[t, y, x] else 2
                    if outage[t, y, x] and low[t, y, x]:
                        touched.add(m)
            for b in touched:
                longest[b] = max(longest[b], run)
            valid = flags == 3
            out[:, y, x] = np.where(valid, longest.astype(np.float32) * np.float32(hours),
                                    np.nan)
    return out


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_run_end_crediting_equals_per_step_crediting(seed):
    rng = np.random.default_rng(seed)
    count, height, width, band_count = 200, 5, 6, 5
    state = rng.random((height, width)) < 0.5
    low = np.zeros((count, height, width), dtype=bool)
    for t in range(count):
        state ^= rng.random((height, width)) < 0.15
        low[t] = state
    outage = rng.random((count, height, width)) < 0.3
    months = rng.integers(-1, band_count, count).astype(np.int32)
    if seed == 1:
        months = np.sort(months)
    fractions = np.where(low, np.float32(0.1), np.float32(0.9)).astype(np.float32)
    margins = np.where(outage, np.float32(-1.0), np.float32(5.0)).astype(np.float32)
    expected = products.safe_haven(fractions, margins, months, band_count,
                                   sunlight_threshold=0.2, earth_threshold_deg=2.0,
                                   time_step_hours=2.5)
    got = _run_end_crediting(low, outage, months, band_count, 2.5)
    np.testing.assert_array_equal(got, expected)
