"""Host-side helpers of the benchmark (CPU): the every-ray distance summary
of two degree batches and the reference arm's measured steps."""

from __future__ import annotations

import numpy as np


def test_distance_over_every_ray_reports_p999_and_max():
    import torch

    import bench

    rng = np.random.default_rng(3)
    a = rng.uniform(-5.0, 30.0, size=(3, 1000, 8)).astype(np.float32)
    b = a.copy()
    # 0.2 % of the rays move by 0.5 deg, one by 2 deg; a shared -inf ray.
    flat = b.reshape(-1)
    moved = rng.choice(flat.size, 48, replace=False)
    flat[moved] += 0.5
    flat[moved[0]] += 1.5
    a[1, 7, 3] = b[1, 7, 3] = -np.inf
    summary = bench.distance_over_every_ray(torch.from_numpy(a), torch.from_numpy(b))
    assert summary["inf_rays_agree"]
    assert summary["rays"] == a.size - 1
    assert abs(summary["max"] - 2.0) < 1e-5
    # 47 of 23,999 rays moved by 0.5: the 99.9th percentile lies among them.
    assert 0.49 < summary["p99.9"] < 0.51
    b[0, 0, 0] = -np.inf
    assert not bench.distance_over_every_ray(torch.from_numpy(a),
                                             torch.from_numpy(b))["inf_rays_agree"]


def test_reference_arm_steps_are_measured(monkeypatch, capsys):
    import json
    import types

    import bench

    class FakeSample:
        threads = 4

        def __init__(self, *args, **kwargs):
            self.calls = 0

        def run(self, rays):
            self.calls += 1
            return 0.5  # seconds per step

    monkeypatch.setattr(bench, "CpuMarchSample", FakeSample)
    monkeypatch.setattr(bench, "build_dems", lambda: (None, None))
    bench.run_reference(types.SimpleNamespace(steps=4, warmup=3))
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["ms_per_step"] == 500.0
    assert line["value"] == bench.REFERENCE_STEP_RAYS / 0.5
    assert line["cpu_baseline"]["cores"] == 4


def test_roofline_reads_the_committed_ncu_summary():
    """The bench's roofline takes the DRAM traffic and the issue-slot share of
    the march from the committed ncu summary of the same workload."""
    import bench

    traffic = bench.profiled_traffic("march_pass_kernel_site_tile.md")
    busy = bench.profiled_value("march_pass_kernel_site_tile.md", "issue_slots_busy")
    assert traffic is not None and 1e8 < traffic < 1e9
    assert busy is not None and 0.5 < busy <= 1.0
    assert bench.profiled_value("march_pass_kernel_site_tile.md", "no_such_key") is None
    assert bench.profiled_traffic("no_such_summary.md") is None
