"""The reference core's remaining oracle free functions on this core's device
code, against the reference core's own outputs recorded in
tests/golden/ref_free.npz (tests/golden/gen_golden_fixtures.py --free):
geometry_project / geometry_tangent (src/bindings.cpp:1859-1889),
geometry_project_batch (:1891-1990), energy_mindet (:2040-2068) and
directional_eval (:1819-1857)."""

from __future__ import annotations

import numpy as np
import pytest

from tests.conftest import GOLDEN
from tests.golden.gen_golden_fixtures import ENTITY_RECORDS

pytestmark = pytest.mark.gpu

_FX = np.load(GOLDEN / "ref_free.npz")
_CON = np.load(GOLDEN / "ref_constrained.npz")
# Feet found by Newton iterations (elliptic arcs, Beziers, B-splines and the
# composite paths holding them) round with each compiler's FMA contraction.
_NEWTON_TAGS = (7, 8, 9, 10, 11)


@pytest.mark.parametrize("tag", sorted(ENTITY_RECORDS))
def test_geometry_project_and_tangent_match_reference(gpu, tag):
    rtol = 1e-10 if tag in _NEWTON_TAGS else 1e-12
    k = f"entity/{tag}/"
    for i in range(len(_CON[k + "pos"])):
        np.testing.assert_allclose(gpu.geometry_project(_CON[k + "pos"][i], tag, _CON[k + "params"]),
                                   _CON[k + "foot"][i], rtol=rtol, atol=1e-15)
    k = f"tangent/{tag}/"
    for i in range(len(_FX[k + "pos"])):
        np.testing.assert_allclose(gpu.geometry_tangent(_FX[k + "pos"][i], tag, _FX[k + "params"]), _FX[k + "t"][i],
                                   rtol=rtol, atol=1e-12)


@pytest.mark.parametrize("k", range(int(_FX["batch/count"])))
def test_geometry_project_batch_matches_reference(gpu, k):
    key = f"batch/{k}/"
    tag = int(_FX[key + "tag"])
    seg = [{"data": _FX[key + f"seg{j}_data"], "off": _FX[key + f"seg{j}_off"]} for j in range(int(_FX[key + "nseg"]))]
    feet, basis = gpu.geometry_project_batch(_FX[key + "q"], tag, _FX[key + "rec"], seg)
    tol = 1e-10 if tag in _NEWTON_TAGS else 1e-12
    assert feet.shape == _FX[key + "feet"].shape and basis.shape == _FX[key + "basis"].shape
    np.testing.assert_allclose(feet, _FX[key + "feet"], rtol=tol, atol=tol)
    np.testing.assert_allclose(basis, _FX[key + "basis"], rtol=tol, atol=tol)


def test_geometry_project_batch_rejects_free_and_unknown_tags(gpu):
    with pytest.raises(ValueError, match="not a projectable"):
        gpu.geometry_project_batch(np.zeros((3, 2)), 0, np.zeros(0), [])
    with pytest.raises(ValueError, match="not a projectable"):
        gpu.geometry_project_batch(np.zeros((3, 3)), 1, np.zeros(4), [])


def test_energy_mindet_matches_reference(gpu):
    import json

    recs = json.loads((GOLDEN / "golden_patch.json").read_text())["records"]
    for r, (e_ref, m_ref) in zip(recs, _FX["energy_mindet"]):
        P, n = int(r["P"]), int(r["n_nodes"])
        e, m = gpu.energy_mindet(np.array(r["X"][: 2 * n]), np.array(r["gc"][:P]), np.array(r["gn0"][:P]),
                                 np.array(r["gn1"][:P]), np.array(r["s0"][:P]), np.array(r["s1"][:P]),
                                 np.array(r["W_inv"][: 4 * P]))
        np.testing.assert_allclose(e, e_ref, rtol=1e-13, atol=1e-14)
        np.testing.assert_allclose(m, m_ref, rtol=1e-13, atol=1e-14)


@pytest.mark.parametrize("d", [2, 3])
def test_directional_eval_matches_reference(gpu, d):
    k = f"dir{d}/"
    e, g = gpu.directional_eval(_FX[k + "X"], _FX[k + "nodes"], _FX[k + "kind"], _FX[k + "ref"], _FX[k + "w"], 1e-3)
    np.testing.assert_allclose(e, float(_FX[k + "e"]), rtol=1e-12)
    np.testing.assert_allclose(g, _FX[k + "g"], rtol=1e-11, atol=1e-12)


def test_directional_eval_rejects_bad_tables(gpu):
    X = np.zeros((4, 2))
    with pytest.raises(ValueError, match="inconsistent sample-table shapes"):
        gpu.directional_eval(X, np.zeros((2, 3), dtype=np.int32), np.zeros(2, dtype=np.int32), np.zeros((2, 2)),
                             np.ones(2))
    with pytest.raises(ValueError, match="unsupported sample kind"):
        gpu.directional_eval(X, np.array([[0, 1, -1, -1]], dtype=np.int32), np.array([7], dtype=np.int32),
                             np.zeros((1, 2)), np.ones(1))
