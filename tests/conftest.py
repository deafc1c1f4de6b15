"""Shared test setup: markers, fixture loading and the oracle build."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and libls200.so")


@pytest.fixture(scope="session", autouse=True)
def _oracle_built():
    import oracle

    oracle.build()


def load_golden(name: str) -> dict:
    with np.load(GOLDEN / name, allow_pickle=False) as archive:
        return {key: archive[key] for key in archive.files}


def pyramid_from(arrays: dict, name: str):
    from lunarscout_b200.contract import PyramidArrays

    return PyramidArrays(
        np.ascontiguousarray(arrays[f"{name}_level0"], dtype=np.float32),
        np.ascontiguousarray(arrays[f"{name}_mips"], dtype=np.float32),
        np.ascontiguousarray(arrays[f"{name}_levels"], dtype=np.int32),
        np.ascontiguousarray(arrays[f"{name}_map"], dtype=np.float32),
        np.ascontiguousarray(arrays[f"{name}_projection"], dtype=np.float32),
    )


@pytest.fixture(scope="session")
def production_case():
    arrays = load_golden("horizon_production.npz")
    pyramids = [pyramid_from(arrays, "dem0"), pyramid_from(arrays, "dem1")]
    return arrays, pyramids


@pytest.fixture(scope="session")
def cuda_session():
    from lunarscout_b200.cuda_backend import CudaSession

    session = CudaSession(0)
    yield session
    session.close()
