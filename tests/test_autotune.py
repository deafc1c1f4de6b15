"""Host logic of the batched-march autotuner: candidate space, selection,
configuration restore and the per-device cache (timings from a fake)."""

from __future__ import annotations

from types import SimpleNamespace

import pytest

from lunarscout_b200.autotune import (
    DEFAULT_CANDIDATES,
    select_best,
    tune_batch,
    workload_key,
)
from lunarscout_b200.cuda_backend import BatchConfig


class FakeSession:
    def __init__(self):
        self.info = SimpleNamespace(name="Fake B200")
        self.config = BatchConfig()
        self.history = []

    def set_batch_config(self, config):
        self.config = config
        self.history.append(config)

    def batch_config(self):
        return self.config


def _fake_run(times):
    def run(session, tiles):
        return times[session.config]
    return run


def test_default_candidates_are_valid_and_unique():
    assert len(set(DEFAULT_CANDIDATES)) == len(DEFAULT_CANDIDATES)
    for config in DEFAULT_CANDIDATES:
        assert config.lanes_per_azimuth in (32, 16, 8, 4, 2, 1)
        assert config.min_blocks in (6, 8)
    assert DEFAULT_CANDIDATES[0] == BatchConfig()


def test_select_best_prefers_the_fastest_then_the_earliest():
    a, b, c = BatchConfig(32), BatchConfig(16), BatchConfig(8)
    assert select_best({a: 2.0, b: 1.0, c: 3.0}, (a, b, c)) == b
    assert select_best({a: 1.0, b: 1.0}, (b, a)) == b
    with pytest.raises(ValueError):
        select_best({}, (a,))


def test_tune_applies_the_winner_or_restores_the_previous():
    session = FakeSession()
    times = {config: 1.0 + i for i, config in enumerate(DEFAULT_CANDIDATES)}
    winner = DEFAULT_CANDIDATES[5]
    times[winner] = 0.5
    result = tune_batch(session, [object()] * 3, device_out=0, run=_fake_run(times))
    assert result.best == winner and session.config == winner
    assert set(result.seconds) == set(DEFAULT_CANDIDATES)
    before = BatchConfig(8, 6)
    session.set_batch_config(before)
    tune_batch(session, [object()], device_out=0, run=_fake_run(times), apply=False)
    assert session.config == before


def test_tune_restores_the_configuration_when_a_run_fails():
    session = FakeSession()
    session.set_batch_config(BatchConfig(16, 8))

    def broken(sess, tiles):
        raise RuntimeError("launch failed")

    with pytest.raises(RuntimeError):
        tune_batch(session, [object()], device_out=0, run=broken)
    assert session.config == BatchConfig(16, 8)


def test_cache_round_trip(tmp_path):
    session = FakeSession()
    cache = tmp_path / "tuning.json"
    times = {config: 2.0 for config in DEFAULT_CANDIDATES}
    times[DEFAULT_CANDIDATES[3]] = 1.0
    first = tune_batch(session, [object()] * 2, device_out=0, run=_fake_run(times),
                       cache_path=cache)
    assert not first.cached and first.key == workload_key("Fake B200", "ladder", 1440, 2)

    def never(sess, tiles):
        raise AssertionError("a cached workload is not timed again")

    second = tune_batch(FakeSession(), [object()] * 2, device_out=0, run=never,
                        cache_path=cache)
    assert second.cached and second.best == DEFAULT_CANDIDATES[3]
    other = tune_batch(FakeSession(), [object()] * 5, device_out=0, run=_fake_run(times),
                       cache_path=cache)
    assert not other.cached
