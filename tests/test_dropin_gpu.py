"""The drop-in boundary, exercised by the reference's own drivers.

tests/golden/ref_dropin.pkl.gz holds every call that the reference's Python
drivers made on ``egg._cpp.cpp_core`` -- ``cpp_structured_sweep`` on the
12-block circle-in-rectangle O-grid, the ``CppStructuredSweepSession`` wrapper
(run, shape+size, get_X, run_fas, mg_levels) on two conforming blocks, the
``cpp_untangle`` delta continuation on a folded O-grid, and the pipeline's
``_cpp_reduce`` energy probe (``egg/smoothing/cpp_backend.py:456-848``,
``egg/pipeline.py:510-527``) -- with the arguments exactly as the drivers
built them and the reference core's results (recorded by
tests/golden/gen_dropin_trace.py).  Each call is replayed here against
``egg_b200.cpp_core`` and its result compared with the reference core's.
"""

from __future__ import annotations

import gzip
import pickle

import numpy as np
import pytest

from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu

with gzip.open(GOLDEN / "ref_dropin.pkl.gz", "rb") as _f:
    _EVENTS = pickle.load(_f)["events"]
SCENARIOS = sorted({ev["scenario"] for ev in _EVENTS})


def _close(got, want, what, rtol, atol):
    if isinstance(want, (tuple, list)):
        assert isinstance(got, (tuple, list)) and len(got) == len(want), (what, got, want)
        for i, (g, w) in enumerate(zip(got, want)):
            _close(g, w, f"{what}[{i}]", rtol, atol)
        return
    if isinstance(want, dict):
        for k, w in want.items():
            _close(got[k], w, f"{what}.{k}", rtol, atol)
        return
    if isinstance(want, (int, str, bool)) or want is None:
        assert got == want, (what, got, want)
        return
    g, w = np.asarray(got, dtype=np.float64), np.asarray(want, dtype=np.float64)
    assert g.shape == w.shape, (what, g.shape, w.shape)
    np.testing.assert_allclose(g, w, rtol=rtol, atol=atol, err_msg=what)


# Tolerances per call: energies, min dets and positions at the trajectory
# tolerances of the other fp64 parity tests; the Newton-footed projections at
# the entity tests' 1e-10.
_TOL = {
    "run": (1e-9, 1e-12),
    "run_fas": (1e-8, 1e-12),
    "get_X": (0.0, 1e-9),
    "cpp_structured_sweep": (1e-9, 1e-9),
    "geometry_project_batch": (1e-10, 1e-12),
}


@pytest.mark.parametrize("scenario", SCENARIOS)
def test_reference_driver_calls_replay(gpu, scenario):
    sessions = {}
    n = 0
    for ev in (e for e in _EVENTS if e["scenario"] == scenario):
        if ev["op"] == "new":
            sessions[ev["sid"]] = gpu.CppStructuredSweepSession(*ev["args"], **ev["kwargs"])
            continue
        target = gpu if ev["op"] == "fn" else sessions[ev["sid"]]
        got = getattr(target, ev["name"])(*ev["args"], **ev["kwargs"])
        rtol, atol = _TOL.get(ev["name"], (1e-12, 1e-12))
        _close(got, ev["result"], f"{scenario}:{ev['name']}#{n}", rtol, atol)
        n += 1
    assert n > 0
