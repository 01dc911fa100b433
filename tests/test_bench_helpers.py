"""Host-side helpers of bench.py (no GPU): the time-to-energy-tolerance band."""

from __future__ import annotations

import bench


def test_sweeps_to_tol_is_the_first_sweep_that_stays_in_the_band():
    E = [10.0, 5.0, 2.0, 1.0000005, 1.0000020, 1.0000001, 1.0]
    # |E - 1| <= 1e-6 from sweep 6 on: sweep 4 is inside but sweep 5 leaves the band
    assert bench._sweeps_to_tol(E, 1.0, 1e-6) == 6
    assert bench._sweeps_to_tol([1.0], 1.0, 1e-6) == 1
    assert bench._sweeps_to_tol([3.0, 1.0], 1.0, 1e-6) == 2


def test_sweeps_to_tol_is_none_when_the_last_report_is_outside():
    assert bench._sweeps_to_tol([3.0, 2.0], 1.0, 1e-6) is None
