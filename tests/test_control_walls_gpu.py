"""Control nets with sliding walls, exercised by the reference's own helpers.

tests/golden/ref_dropin_walls.pkl.gz holds every call that the reference's
wall-session helpers (``tests/smoothing/test_control_wall_cpp.py``, over
``egg/smoothing/control_backend.py`` ``build_control_wire(..., walls=)``)
made on ``egg._cpp.cpp_core``: an arc wall with the orthogonality dial off,
a sheared arc wall in the off, penalty and hard modes with exact PCG solves,
the hard mode again with the default inexact solves, and a 3D cube whose
bottom face slides on a sphere (off and hard).  Each call is replayed on
``egg_b200.cpp_core`` and compared with the reference core's result
(recorded by ``tests/golden/gen_dropin_trace.py --walls``).  The frames
(projections, tangents, hard-leg snap, Boolean-sum re-extension) are rebuilt
on the host every outer iteration, as the reference does.
"""

from __future__ import annotations

import numpy as np
import pytest

from tests import control_replay

pytestmark = pytest.mark.gpu

_EVENTS = control_replay.load("ref_dropin_walls.pkl.gz")
SCENARIOS = sorted({ev["scenario"] for ev in _EVENTS})


# The sphere wall's face centre sits on the sphere's pole, where the
# latitude chart lat = asin(m . az) of the entity's projection amplifies a
# last-bit difference about 1 / sqrt(1 - x^2) ~ 7e7-fold: both cores project
# the centre node with ~1e-8 of rounding noise, and their host arithmetic
# orders differ in the last bits (the frames here and the reference's agree
# to ~10 ulp elsewhere).  With the default inexact PCG the hard legs' snap
# compounds it over the run.  The arc walls have no such point and match at
# the trajectory tolerances.
_TOL = {"sphere_off": (1e-6, 1e-7), "sphere_hard": (1e-4, 1e-4)}


@pytest.mark.parametrize("scenario", SCENARIOS)
def test_reference_wall_session_replay(gpu, scenario):
    rtol, x_atol = _TOL.get(scenario, (control_replay.RTOL, 1e-10))
    assert control_replay.replay(gpu, _EVENTS, scenario, rtol=rtol, x_atol=x_atol) > 0


def _new(gpu, scenario):
    ev = next(e for e in _EVENTS if e["scenario"] == scenario and e["op"] == "new")
    return ev, gpu.CppStructuredSweepSession(*ev["args"], **ev["kwargs"])


def test_wall_rows_stay_on_the_arc(gpu):
    """After a run the wall-row nodes lie on the wall's entity: the closing
    frame re-extends b against the projected spline boundary."""
    ev, s = _new(gpu, "arc_off")
    s.run_control(5)
    ctl = ev["kwargs"]["control"]
    w = ctl["walls"][0]
    cx, cy, r = (float(v) for v in np.asarray(w["params"])[:3])
    shape = [len(ctl[f"off{k}"]) for k in range(2)]
    bgd = np.asarray(ev["args"][1]["block_global_dof"]).reshape(shape)
    X = s.get_X().reshape(-1, 2)
    ids = bgd[:, 0] if w["axis"] == 1 else bgd[0, :]
    rad = np.hypot(X[ids, 0] - cx, X[ids, 1] - cy)
    np.testing.assert_allclose(rad, r, rtol=1e-12)


def test_segmented_wall_entity_is_refused(gpu):
    ev, _ = _new(gpu, "arc_off")
    ctl = dict(ev["kwargs"]["control"])
    ctl["walls"] = [dict(ctl["walls"][0], tag=10)]
    with pytest.raises(NotImplementedError, match="segmented"):
        gpu.CppStructuredSweepSession(*ev["args"], **{**ev["kwargs"], "control": ctl})
    ctl["walls"] = [dict(ctl["walls"][0], tag=13)]  # a 3D line in a 2D session
    with pytest.raises(ValueError, match="tangent dimension"):
        gpu.CppStructuredSweepSession(*ev["args"], **{**ev["kwargs"], "control": ctl})


def test_wall_control_outside_the_free_set_is_refused(gpu):
    ev, _ = _new(gpu, "arc_off")
    ctl = dict(ev["kwargs"]["control"])
    w = ctl["walls"][0]
    fixed = np.setdiff1d(np.arange(len(ctl["C0"]) // 2), ctl["free_idx"])
    p0 = np.asarray(w["p0"]).copy()
    p0[0] = fixed[0]
    ctl["walls"] = [dict(w, p0=p0)]
    with pytest.raises(ValueError, match="not in the free set"):
        gpu.CppStructuredSweepSession(*ev["args"], **{**ev["kwargs"], "control": ctl})
