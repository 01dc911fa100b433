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

import gzip
import pickle

import numpy as np
import pytest

from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu

with gzip.open(GOLDEN / "ref_dropin_topo.pkl.gz", "rb") as _f:
    _EVENTS = pickle.load(_f)["events"]
SCENARIOS = sorted({ev["scenario"] for ev in _EVENTS})

# Energies, min dets, step lengths, lattice and positions at the trajectory
# tolerances of the other fp64 control tests.  A PCG solve that stops at
# rtol may take one or two iterations more or fewer when its dot products
# round differently, so its iteration count is compared to within two and its
# final relative residual to within one decade.
_RTOL, _ATOL = 1e-9, 1e-12


def _check_report(got, want, what):
    for k in ("energies", "mindets", "alphas"):
        g, w = np.asarray(got[k]), np.asarray(want[k])
        assert g.shape == w.shape, (what, k, g, w)
        np.testing.assert_allclose(g, w, rtol=_RTOL, atol=_ATOL, err_msg=f"{what}.{k}")
    assert got["iters"] == want["iters"] and bool(got["converged"]) == bool(want["converged"]), (what, got, want)
    assert len(got["frame_jumps"]) == len(want["frame_jumps"]) == 0
    gi, wi = np.asarray(got["pcg_iters"]), np.asarray(want["pcg_iters"])
    assert gi.shape == wi.shape, (what, gi, wi)
    assert np.all(np.abs(gi - wi) <= 2), (what, gi, wi)
    gr, wr = np.asarray(got["pcg_relres"]), np.asarray(want["pcg_relres"])
    assert gr.shape == wr.shape
    pos = wr > 0
    assert np.all(gr[~pos] == 0.0)
    assert np.all(np.abs(np.log10(gr[pos] / wr[pos])) <= 1.0), (what, gr, wr)


@pytest.mark.parametrize("scenario", SCENARIOS)
def test_reference_topology_driver_replay(gpu, scenario):
    sessions = {}
    n = 0
    for ev in (e for e in _EVENTS if e["scenario"] == scenario):
        if ev["op"] == "new":
            sessions[ev["sid"]] = gpu.CppStructuredSweepSession(*ev["args"], **ev["kwargs"])
            continue
        got = getattr(sessions[ev["sid"]], ev["name"])(*ev["args"], **ev["kwargs"])
        what = f"{scenario}:{ev['name']}#{n}"
        if ev["name"] == "run_control":
            _check_report(got, ev["result"], what)
        elif ev["name"] in ("get_C", "get_X"):
            np.testing.assert_allclose(got, ev["result"], rtol=_RTOL, atol=1e-10, err_msg=what)
        else:
            assert got is None and ev["result"] is None, what
        n += 1
    assert n > 0


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
