"""The wire builders reproduce the reference's wire format exactly."""

from __future__ import annotations

import numpy as np

from egg_b200 import configs, wire
from tests.conftest import GOLDEN

_W = np.load(GOLDEN / "ref_wire_disk_oh17.npz")


def test_flat_wire_matches_reference_builder():
    g = configs.disk_oh(17, frac=0.25, seed=2)
    for tag, w in (("eye", np.eye(2)), ("aniso", np.array([[1.0, 0.2], [0.0, 1.3]]))):
        ctx = wire.flat_wire(g.blocks, g.free, 2, w_inv=w)
        for k, v in ctx["groups"][0].items():
            if isinstance(v, np.ndarray):
                np.testing.assert_array_equal(np.asarray(v).reshape(-1), _W[f"{tag}/group/{k}"].reshape(-1), k)
        for k, v in ctx["energy_stencil"].items():
            if isinstance(v, np.ndarray):
                np.testing.assert_array_equal(np.asarray(v).reshape(-1), _W[f"{tag}/es/{k}"].reshape(-1), k)


def test_structured_tables_match_reference_builder():
    g = configs.disk_oh(17, frac=0.25, seed=2)
    st = wire.structured_tables(g.blocks)
    for k, v in st.items():
        if isinstance(v, list):
            for i, a in enumerate(v):
                np.testing.assert_array_equal(np.asarray(a), _W[f"st/{k}/{i}"])
        else:
            np.testing.assert_array_equal(np.asarray(v), _W[f"st/{k}"])


def test_wire_invariants():
    g = configs.disk_oh(9)
    grp = g.wire()["groups"][0]
    assert grp["P_of"].sum() == grp["gc"].size
    assert set(np.unique(grp["role"])) <= {-1, 0, 1, 2}
    interior = grp["interior_block"] >= 0
    assert (grp["P_of"][interior] == 0).all() and (grp["P_of"][~interior] > 0).all()
    # every stored DOF owns at least its corner samples
    es = g.wire()["energy_stencil"]
    assert es["num_samples"] == sum(4 * (b.shape[0] - 1) * (b.shape[1] - 1) for b in g.blocks)


def test_compact_wire_drops_stencil_arrays():
    g = configs.unit_square(17)
    full, comp = g.wire(), g.wire(compact=True)
    assert comp["energy_stencil"]["structured"] == 1
    assert "gc" not in comp["energy_stencil"]
    assert comp["energy_stencil"]["num_samples"] == full["energy_stencil"]["num_samples"]
    for k in ("dof_idx", "P_of", "interior_block", "role"):
        np.testing.assert_array_equal(full["groups"][0][k], comp["groups"][0][k])


def test_configs_are_deterministic_and_valid():
    a, b = configs.disk_oh(17, seed=3), configs.disk_oh(17, seed=3)
    np.testing.assert_array_equal(a.X, b.X)
    assert configs.grid_mindet(a.blocks, a.X).min() > 0
    t = configs.tangled_square(65, seed=1)
    assert 0.05 <= t.meta["inverted_cell_fraction"] < 0.1
    s = configs.unit_square(33, frac=0.3, seed=0)
    assert s.num_free == 31 * 31
