"""B-spline / NURBS surfaces (entity tag 14): constrained DOFs sliding on
them, against the reference core.

The unit cube of ``configs.cube_bsurf`` has its top face on a bicubic
B-spline bump and its face x ~ 1 on a rational biquadratic NURBS sheet.
``tests/golden/ref_bsurf.npz`` (``gen_golden_fixtures.py --bsurf``) holds the
reference core's sweeps (barrier at omega 1 and 0.8, shape+size), a session
run in two calls (the seeds persist: each call's first sweep projects from
them in world space, later sweeps search in the surface parameters), FAS
V-cycles, and its batched projection onto a polynomial, a rational and a
UV-trimmed surface.  The feet come from Newton iterations, which round with
each compiler's FMA contraction: positions are compared at 1e-10 of the
smallest edge, as the other Newton-footed entities are.
"""

from __future__ import annotations

import numpy as np
import pytest

from egg_b200 import configs
from tests.conftest import GOLDEN
from tests.golden.gen_golden_fixtures import BSURF_CASE, BSURF_RUNS, bsurf_entities

pytestmark = pytest.mark.gpu

_FX = np.load(GOLDEN / "ref_bsurf.npz")


def _grid():
    return getattr(configs, BSURF_CASE[0])(**BSURF_CASE[1])


def _hmin(g):
    return float(configs._min_edge(g.blocks, g.X).min())


def _session(gpu, g, **kw):
    return gpu.CppStructuredSweepSession(g.wire(), g.structured(), g.X_flat(), dim=3, **kw)


@pytest.mark.parametrize("run", BSURF_RUNS, ids=lambda r: f"{r[0]}-{r[2]}")
def test_bsurf_sweeps_match_reference(gpu, run):
    phase, delta, omega, n = run
    g = _grid()
    key = f"{phase}/{omega}"
    s = _session(gpu, g)
    s.run(1, phase=phase, delta=delta, omega=omega)
    assert np.abs(s.get_X() - _FX[key + "/X1"]).max() <= 1e-10 * _hmin(g)
    s2 = _session(gpu, g)
    E, M = s2.run(n, phase=phase, delta=delta, omega=omega, report_every=1)
    np.testing.assert_allclose(E, _FX[key + "/E"], rtol=1e-9)
    np.testing.assert_allclose(M, _FX[key + "/M"], rtol=1e-8, atol=1e-16)
    assert np.abs(s2.get_X() - _FX[key + "/Xn"]).max() <= 1e-9 * _hmin(g)


def test_bsurf_seeds_persist_across_calls(gpu):
    g = _grid()
    s = _session(gpu, g)
    e_a, _ = s.run(5, report_every=1)
    e_b, _ = s.run(10, report_every=1)
    np.testing.assert_allclose(np.concatenate([e_a, e_b]), _FX["twocalls/E"], rtol=1e-9)
    assert np.abs(s.get_X() - _FX["twocalls/X"]).max() <= 1e-9 * _hmin(g)


def test_bsurf_fas_matches_reference(gpu):
    g = _grid()
    s = _session(gpu, g)
    E, M = s.run_fas(3, nu_pre=2, nu_post=2, nu_coarse=16, omega=1.0, max_levels=32, phase="barrier")
    np.testing.assert_allclose(E, _FX["fas/E"], rtol=1e-8)
    np.testing.assert_allclose(M, _FX["fas/M"], rtol=1e-7)
    assert np.abs(s.get_X() - _FX["fas/X"]).max() <= 1e-9 * _hmin(g)


@pytest.mark.parametrize("name", ["poly", "nurbs", "trimmed"])
def test_bsurf_projection_matches_reference(gpu, name):
    ent = {n: (t, r, s) for n, t, r, s in bsurf_entities()}[name]
    tag, rec, seg = ent
    feet, basis = gpu.geometry_project_batch(_FX[f"project/{name}/q"], tag, rec, seg)
    # the foot iterations stop once the parameter moves less than 1e-9, so a
    # foot is fixed to about that much of |S_u|, |S_v| (~1)
    np.testing.assert_allclose(feet, _FX[f"project/{name}/foot"], rtol=0, atol=1e-8)
    np.testing.assert_allclose(basis, _FX[f"project/{name}/basis"], rtol=0, atol=1e-7)


def test_bsurf_nodes_stay_on_their_surfaces(gpu):
    g = _grid()
    s = _session(gpu, g)
    s.run(10)
    X = s.get_X().reshape(-1, 3)
    ids = np.array(sorted(g.constraints))
    X0 = g.X.reshape(-1, 3)
    moved = 0
    for v in ids:
        if np.array_equal(X[v], X0[v]):
            continue  # never accepted a trial: still at its (off-surface) start
        moved += 1
        t, r, sg = g.constraints[int(v)]
        sd = [{"data": np.asarray(a, dtype=np.float64), "off": np.array([0, np.asarray(a).size], np.int32)}
              for a in sg]
        foot, _ = gpu.geometry_project_batch(X[v][None, :], t, np.asarray(r), sd)
        assert np.abs(foot[0] - X[v]).max() <= 1e-9
    assert moved > len(ids) // 2
