"""Replay of recorded reference-driver calls on control sessions (shared by
the topology and wall tests).

A trace is a list of events recorded by tests/golden/gen_dropin_trace.py:
``new`` (the session constructor with its wire) and ``call`` (a method with
its arguments and the reference core's result).  Reports of ``run_control``
are compared field by field: energies, min dets, step lengths, iteration
count and convergence at the trajectory tolerances of the other fp64 control
tests.  A PCG solve that stops at rtol may take a few iterations more or
fewer when its dot products round differently, so its iteration count is
compared to within two or 5%, whichever is larger (four or 25% for the
inexact solves of a forcing run), and its final relative residual to within
one decade.
"""

from __future__ import annotations

import gzip
import pickle

import numpy as np

from tests.conftest import GOLDEN

RTOL, ATOL = 1e-9, 1e-12


def load(name: str) -> list[dict]:
    with gzip.open(GOLDEN / name, "rb") as f:
        return pickle.load(f)["events"]


def check_report(got, want, what, rtol=RTOL, atol=ATOL, forcing=False):
    for k in ("energies", "mindets", "alphas"):
        g, w = np.asarray(got[k]), np.asarray(want[k])
        assert g.shape == w.shape, (what, k, g, w)
        np.testing.assert_allclose(g, w, rtol=rtol, atol=atol, err_msg=f"{what}.{k}")
    assert got["iters"] == want["iters"] and bool(got["converged"]) == bool(want["converged"]), (what, got, want)
    fg, fw = np.asarray(got["frame_jumps"]), np.asarray(want["frame_jumps"])
    assert fg.shape == fw.shape, (what, fg, fw)
    # a frame's jump is a difference of two energies: absolute at their scale
    scale = float(np.abs(np.asarray(want["energies"])).max()) if len(want["energies"]) else 1.0
    np.testing.assert_allclose(fg, fw, rtol=0, atol=rtol * scale + atol, err_msg=f"{what}.frame_jumps")
    gi, wi = np.asarray(got["pcg_iters"]), np.asarray(want["pcg_iters"])
    assert gi.shape == wi.shape, (what, gi, wi)
    # an inexact solve (forcing: stop at a relative residual up to 0.5) stops
    # wherever its residual first crosses a loose bound, so its count moves
    # further with the same rounding
    slack = np.maximum(4, 0.25 * wi) if forcing else np.maximum(2, 0.05 * wi)
    assert np.all(np.abs(gi - wi) <= slack), (what, gi, wi)
    gr, wr = np.asarray(got["pcg_relres"]), np.asarray(want["pcg_relres"])
    assert gr.shape == wr.shape
    pos = wr > 0
    assert np.all(gr[~pos] == 0.0)
    assert np.all(np.abs(np.log10(gr[pos] / wr[pos])) <= 1.0), (what, gr, wr)


def _close(got, want, what, rtol, atol):
    if isinstance(want, (tuple, list)):
        assert isinstance(got, (tuple, list)) and len(got) == len(want), (what, got, want)
        for i, (g, w) in enumerate(zip(got, want)):
            _close(g, w, f"{what}[{i}]", rtol, atol)
        return
    g, w = np.asarray(got, dtype=np.float64), np.asarray(want, dtype=np.float64)
    assert g.shape == w.shape, (what, g.shape, w.shape)
    np.testing.assert_allclose(g, w, rtol=rtol, atol=atol, err_msg=what)


def replay(core, events, scenario, rtol=RTOL, atol=ATOL, x_atol=1e-10):
    """Replay one scenario's calls on `core`; returns the number compared.
    Free-function calls of the driver (entity projections) are compared at
    the entity tests' 1e-10."""
    sessions = {}
    n = 0
    for ev in (e for e in events if e["scenario"] == scenario):
        if ev["op"] == "new":
            sessions[ev["sid"]] = core.CppStructuredSweepSession(*ev["args"], **ev["kwargs"])
            continue
        if ev["op"] == "fn":
            got = getattr(core, ev["name"])(*ev["args"], **ev["kwargs"])
            _close(got, ev["result"], f"{scenario}:{ev['name']}#{n}", 1e-10, 1e-12)
            n += 1
            continue
        got = getattr(sessions[ev["sid"]], ev["name"])(*ev["args"], **ev["kwargs"])
        what = f"{scenario}:{ev['name']}#{n}"
        if ev["name"] == "run_control":
            check_report(got, ev["result"], what, rtol, atol, forcing=ev["kwargs"].get("pcg_forcing", True))
        elif ev["name"] in ("get_C", "get_X"):
            np.testing.assert_allclose(got, ev["result"], rtol=rtol, atol=x_atol, err_msg=what)
        else:
            assert got is None and ev["result"] is None, what
        n += 1
    return n
