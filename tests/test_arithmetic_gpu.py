"""The march's reciprocal (hardware approximation plus one Newton-Raphson
correction) equals the IEEE round-to-nearest reciprocal on every pattern it
can receive (|x| >= 2^-64, both signs), on this device: the premise of the
march's bit parity with the reference, whose Numba-CUDA kernel divides with
IEEE rounding."""

from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu


def test_reciprocal_matches_ieee_on_every_pattern(cuda_session):
    mismatches, checked = cuda_session.check_arithmetic()
    assert mismatches == 0
    assert checked == 2 * (0x80000000 - (63 << 23))
