"""Multi-block control topologies, exercised by the reference's own driver.

tests/golden/ref_dropin_topo.pkl.gz holds every call that the reference's
``run_control_topo`` (``egg/smoothing/control_backend.py:646``) made on
``egg._cpp.cpp_core`` for the reference's multi-block control test grids
(``tests/smoothing/test_control_topology.py``): a two-block seam with a wavy
edge, a 2 x 2 crossing, a valence-3 fan, a C2-penalty seam, a seam with
per-iteration orthogonality penalty uploads, and an inexact-Newton crossing.
Each call -- the session constructor with the ``control['blocks']`` wire,
``run_control``, ``get_C``, ``set_control_penalty``, ``get_X`` -- is replayed
against ``egg_b200.cpp_core`` and its result compared with the reference
core's (recorded by ``tests/golden/gen_dropin_trace.py --topo``).
"""

from __future__ import annotations

import numpy as np
import pytest

from tests import control_replay

pytestmark = pytest.mark.gpu

_EVENTS = control_replay.load("ref_dropin_topo.pkl.gz")
SCENARIOS = sorted({ev["scenario"] for ev in _EVENTS})


@pytest.mark.parametrize("scenario", SCENARIOS)
def test_reference_topology_driver_replay(gpu, scenario):
    assert control_replay.replay(gpu, _EVENTS, scenario) > 0


def _topo_session(gpu, scenario="seam"):
    ev = next(e for e in _EVENTS if e["scenario"] == scenario and e["op"] == "new")
    return ev, gpu.CppStructuredSweepSession(*ev["args"], **ev["kwargs"])


def test_set_control_b_moves_only_that_net(gpu):
    ev, s = _topo_session(gpu)
    ctl = ev["kwargs"]["control"]
    X_wire = s.get_X().copy()
    b0 = np.asarray(ctl["blocks"][1]["b"], dtype=np.float64)
    s.set_control_b(1, b0 + 0.0)  # evaluates the nets: X = M C0 + b
    X0 = s.get_X().copy()
    assert np.abs(X0 - X_wire).max() > 0  # the constructor left the wire's X
    s.set_control_b(1, b0 + 0.0)
    np.testing.assert_array_equal(s.get_X(), X0)
    s.set_control_b(1, b0 + 1e-3)
    moved = np.abs(s.get_X() - X0) > 0
    assert moved.any() and not moved.all()
    with pytest.raises(ValueError, match="set_b block index out of range"):
        s.set_control_b(2, b0)
    with pytest.raises(ValueError, match="set_b size mismatch"):
        s.set_control_b(0, b0[:-2])


def test_setters_validate_like_the_reference(gpu):
    ev, s = _topo_session(gpu)
    ctl = ev["kwargs"]["control"]
    nsd = len(ctl["C0"])
    off, col, coef = (np.asarray(ctl[k]) for k in ("r_off", "r_col", "r_coef"))
    with pytest.raises(ValueError, match="reduction row count"):
        s.set_control_reduction(int(ctl["nq"]), off[:-1], col, coef)
    with pytest.raises(ValueError, match="reduction column out of range"):
        s.set_control_reduction(int(col.max()), off, col, coef)
    with pytest.raises(ValueError, match="penalty weight count"):
        s.set_control_penalty(np.array([0, 1]), np.array([0]), np.array([1.0]), np.array([1.0, 2.0]))
    with pytest.raises(ValueError, match="penalty column out of range"):
        s.set_control_penalty(np.array([0, 1]), np.array([nsd]), np.array([1.0]), np.array([1.0]))
    # a rejected call leaves the topology as it was: the same run as a fresh session
    fresh = _topo_session(gpu)[1]
    a, b = s.run_control(3, pcg_forcing=False, pcg_rtol=1e-12, pcg_max_iter=2000), \
        fresh.run_control(3, pcg_forcing=False, pcg_rtol=1e-12, pcg_max_iter=2000)
    np.testing.assert_array_equal(a["energies"], b["energies"])


def test_reduction_replacement_keeps_its_row_space(gpu):
    """Replacing R by the same CSR reproduces the run; pinning the reduced
    unknowns (R = 0) leaves the lattice where it is."""
    ev, s = _topo_session(gpu)
    ctl = ev["kwargs"]["control"]
    off, col, coef = (np.asarray(ctl[k]) for k in ("r_off", "r_col", "r_coef"))
    s.set_control_reduction(int(ctl["nq"]), off, col, coef)
    fresh = _topo_session(gpu)[1]
    kw = dict(pcg_forcing=False, pcg_rtol=1e-12, pcg_max_iter=2000)
    np.testing.assert_array_equal(s.run_control(2, **kw)["energies"], fresh.run_control(2, **kw)["energies"])
    C = s.get_C().copy()
    s.set_control_reduction(0, np.zeros(len(C) + 1, dtype=np.int32), np.zeros(0, dtype=np.int32), np.zeros(0))
    rep = s.run_control(5, **kw)
    assert rep["iters"] == 0 and len(rep["energies"]) == 1
    np.testing.assert_array_equal(s.get_C(), C)
