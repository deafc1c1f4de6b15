"""Recycled page-locked result arrays of the march calls."""

from __future__ import annotations

import gc

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_pool_recycles_a_dropped_buffer_and_keeps_live_ones_apart(cuda_session):
    from lunarscout_b200._native import PinnedPool

    pool = PinnedPool(keep=1)
    first = pool.empty((64, 1440), np.float32)
    address = first.ctypes.data
    first[:] = 1.0
    second = pool.empty((64, 1440), np.float32)
    assert second.ctypes.data != address
    second[:] = 2.0
    assert float(first.sum()) == 64 * 1440
    del first
    gc.collect()
    third = pool.empty((64, 1440), np.float32)
    assert third.ctypes.data == address
    assert third.flags.writeable and third.flags.c_contiguous
    view = third[3:5]
    del third
    gc.collect()
    fourth = pool.empty((64, 1440), np.float32)
    assert fourth.ctypes.data != address  # a live view keeps its buffer
    view[:] = 7.0
    assert float(view.sum()) == 7.0 * 2 * 1440
