"""Host-side helpers of bench.py."""

from __future__ import annotations

import bench


def test_first_at_is_the_first_report_at_or_below_the_target():
    E = [5.0, 3.0, 1.000002, 1.0000005, 0.9, 1.2]
    assert bench._first_at(E, 1.0, 1e-6) == 4
    assert bench._first_at([1.0], 1.0, 1e-6) == 1
    assert bench._first_at([-2.0, -3.0], -3.0, 1e-6) == 2


def test_first_at_is_none_when_no_report_reaches_the_target():
    assert bench._first_at([3.0, 2.0], 1.0, 1e-6) is None
