"""Soft-term wire tables (no GPU): the per-DOF directional and curvature
tables and the whole-sample directional table that ``egg_b200.wire`` emits
equal the reference's own builders' output for the same terms
(``egg/smoothing/directional.py:381-459``,
``egg/smoothing/interface_c2.py:233-279``; recorded in ref_soft.npz)."""

from __future__ import annotations

import numpy as np
import pytest

from tests.conftest import GOLDEN
from tests.golden.gen_golden_fixtures import CASES_SOFT, case_grid

_FX = np.load(GOLDEN / "ref_soft.npz")


@pytest.mark.parametrize("case", sorted(CASES_SOFT))
def test_soft_tables_match_reference_builders(case):
    g = case_grid(case)
    w = g.wire()
    grp, es = w["groups"][0], w["energy_stencil"]
    seen = 0
    for part, src in (("dof", grp), ("dof_curv", grp), ("es", es)):
        for key in [k for k in _FX.files if k.startswith(f"table/{case}/{part}/")]:
            name = key.rsplit("/", 1)[1]
            np.testing.assert_array_equal(np.asarray(src[name]).ravel(), _FX[key].ravel(), err_msg=key)
            seen += 1
    assert seen == (19 if g.d == 2 else 15)
    # every soft term names the DOF in its listed slot
    K = grp["dir_k"]
    nodes = grp["dir_nodes"].reshape(-1, K, 4)
    slot = grp["dir_slot"].reshape(-1, K)
    for i, dof in enumerate(grp["dof_idx"]):
        for j in range(K):
            if slot[i, j] >= 0:
                assert nodes[i, j, slot[i, j]] == dof


def test_soft_tables_absent_without_terms():
    g = case_grid("square_soft17")
    g.soft = {}
    w = g.wire()
    assert "dir_k" not in w["groups"][0] and "curv_k" not in w["groups"][0]
    assert "dir_num" not in w["energy_stencil"]


@pytest.mark.parametrize("key, cut", [("dir_nodes", 1), ("dir_ref", 2), ("dir_weight", 1), ("curv_slot", 1),
                                      ("curv_weight", 3)])
def test_malformed_soft_tables_are_refused_before_the_device(core, key, cut):
    g = case_grid("square_soft17")
    w = g.wire()
    w["groups"][0][key] = w["groups"][0][key][:-cut]
    with pytest.raises(ValueError, match=key):
        core.CppStructuredSweepSession(w, g.structured(), g.X_flat())


def test_malformed_whole_sample_table_is_refused(core):
    g = case_grid("square_soft17")
    w = g.wire()
    w["energy_stencil"]["dir_kind"] = w["energy_stencil"]["dir_kind"][:-1]
    with pytest.raises(ValueError, match="dir_kind"):
        core.CppStructuredSweepSession(w, g.structured(), g.X_flat())
    w = g.wire()
    w["groups"][0]["dir_k"] = -1
    with pytest.raises(ValueError, match="dir_k"):
        core.CppStructuredSweepSession(w, g.structured(), g.X_flat())
