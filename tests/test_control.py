"""Control-net reduced Gauss-Newton.

CPU: egg_b200.control rebuilds the reference's control wires (B-spline
bases, facet fit, Boolean-sum offset, bands) from the same block nodes, and
malformed wires are refused before any device is touched.

GPU: run_control against the reference core's own run_control (shim build,
fp64) and against the reference's NumPy dense reduced-GN oracle
(reference tests/smoothing/test_control_cpp.py), set_C / get_C, nodal
interop, and a batch of nets against separate sessions."""

from __future__ import annotations

import numpy as np
import pytest

from egg_b200 import configs, control
from tests.conftest import GOLDEN
from tests.golden.gen_golden_fixtures import CONTROL_CASES, control_case_grid

_FX = np.load(GOLDEN / "ref_control.npz")


def _wire(name):
    pre = f"{name}/wire/"
    w = {k[len(pre):]: _FX[k] for k in _FX.files if k.startswith(pre)}
    w["block"] = int(w["block"])
    w["k_supp"] = int(w["k_supp"])
    return w


def _grid(name):
    return control_case_grid(name, _FX)


# ---------------------------------------------------------------- CPU ----


@pytest.mark.parametrize("name", list(CONTROL_CASES))
def test_wire_builder_matches_reference(name):
    g = _grid(name)
    blk = CONTROL_CASES[name][3]
    ref = _wire(name)
    w = control.control_wire(control.grid_block_nodes(g, blk), CONTROL_CASES[name][2], block=blk)
    assert w["k_supp"] == ref["k_supp"] and w["block"] == ref["block"]
    np.testing.assert_array_equal(w["ctrl_shape"], ref["ctrl_shape"])
    np.testing.assert_array_equal(w["free_idx"], ref["free_idx"])
    for k in range(g.d):
        np.testing.assert_array_equal(w[f"off{k}"], ref[f"off{k}"])
        np.testing.assert_allclose(w[f"wt{k}"], ref[f"wt{k}"], rtol=0, atol=1e-15)
    scale = np.abs(g.X).max()
    np.testing.assert_allclose(w["C0"], ref["C0"], rtol=0, atol=1e-12 * scale)
    np.testing.assert_allclose(w["b"], ref["b"], rtol=0, atol=1e-12 * scale)


def test_prolong_plus_offset_reproduces_the_block():
    g = configs.unit_cube(7, frac=0.15, seed=3)
    X0 = control.grid_block_nodes(g, 0)
    bases = control.axis_bases(X0.shape[:-1], (4, 5, 4))
    C = control.fit_lattice(bases, X0)
    b = control.boolean_sum_offset(bases, C, X0)
    X = control.prolong(bases, C) + b
    bm = control.boundary_mask(X0.shape[:-1])
    np.testing.assert_allclose(X[bm], X0[bm], atol=1e-13)


def _session_args(name):
    g = _grid(name)
    return g, (g.wire(), g.structured(), g.X_flat())


@pytest.mark.parametrize("bad, match", [
    (lambda w: {k: v for k, v in w.items() if k != "C0"}, "missing key"),
    (lambda w: {**w, "ctrl_shape": np.array([6], dtype=np.int32)}, "ctrl_shape"),
    (lambda w: {**w, "wt0": w["wt0"][:-1]}, "wt0 size"),
    (lambda w: {**w, "C0": w["C0"][:-2]}, "C0 size"),
])
def test_malformed_wire_is_refused_before_the_device(core, bad, match):
    g, (ctx, st, X) = _session_args("wavy9")
    with pytest.raises(ValueError, match=match):
        core.CppStructuredSweepSession(ctx, st, X, control=bad(_wire("wavy9")))


def _walls_new():
    """The constructor call of the reference's arc-wall session
    (tests/golden/ref_dropin_walls.pkl.gz)."""
    import gzip
    import pickle

    from tests.conftest import GOLDEN

    with gzip.open(GOLDEN / "ref_dropin_walls.pkl.gz", "rb") as f:
        ev = next(e for e in pickle.load(f)["events"] if e["scenario"] == "arc_off" and e["op"] == "new")
    return ev["args"], ev["kwargs"]


def _with_wall(ctl, **kv):
    return {**ctl, "walls": [dict(ctl["walls"][0], **kv)]}


@pytest.mark.parametrize("bad, match", [
    (lambda c: {k: v for k, v in c.items() if k != "X0"}, "walls require X0"),
    (lambda c: {**c, "X0": np.asarray(c["X0"])[:-2]}, "X0 size"),
    (lambda c: _with_wall(c, axis=2), "axis/side/mode"),
    (lambda c: _with_wall(c, mode=3), "axis/side/mode"),
    (lambda c: _with_wall(c, weight=np.zeros(1)), "p0/p1/weight length mismatch"),
    (lambda c: _with_wall(c, p1=np.full(len(c["walls"][0]["p1"]), 10**6, dtype=np.int32)), "control id out of range"),
])
def test_malformed_wall_wire_is_refused_before_the_device(core, bad, match):
    args, kwargs = _walls_new()
    with pytest.raises(ValueError, match=match):
        core.CppStructuredSweepSession(*args, **{**kwargs, "control": bad(kwargs["control"])})


def test_batch_refuses_walls(core):
    args, kwargs = _walls_new()
    with pytest.raises(NotImplementedError, match="walls"):
        core.CppBatchSweepSession([tuple(args)], dim=kwargs["dim"], control=[kwargs["control"]])


def _topo_new():
    """The constructor call the reference's run_control_topo made for its
    two-block seam grid (tests/golden/ref_dropin_topo.pkl.gz)."""
    import gzip
    import pickle

    from tests.conftest import GOLDEN

    with gzip.open(GOLDEN / "ref_dropin_topo.pkl.gz", "rb") as f:
        ev = next(e for e in pickle.load(f)["events"] if e["scenario"] == "seam" and e["op"] == "new")
    return ev["args"], ev["kwargs"]


def _with_block(ctl, i, **kv):
    blocks = [dict(b) for b in ctl["blocks"]]
    blocks[i].update(kv)
    return {**ctl, "blocks": blocks}


@pytest.mark.parametrize("bad, exc, match", [
    (lambda c: _with_block(c, 1, ctrl_shape=np.array([1, 6], dtype=np.int32)), ValueError, "ctrl_shape entry"),
    (lambda c: _with_block(c, 0, wt0=np.asarray(c["blocks"][0]["wt0"])[:-1]), ValueError, "wt0 size"),
    (lambda c: _with_block(c, 0, k_supp=0), ValueError, "k_supp"),
    (lambda c: _with_block(c, 1, b=np.asarray(c["blocks"][1]["b"])[:-2]), ValueError, "b size"),
    (lambda c: _with_block(c, 1, X0=np.zeros(3)), ValueError, "X0 size"),
    (lambda c: {**c, "C0": np.asarray(c["C0"])[:-2]}, ValueError, "C0 size"),
    (lambda c: {**c, "r_off": np.asarray(c["r_off"])[:-1]}, ValueError, "malformed reduction CSR"),
    (lambda c: {**c, "p_off": np.array([0, 1]), "p_col": np.array([0]), "p_coef": np.array([1.0]),
                "p_w": np.array([1.0, 1.0])}, ValueError, "malformed penalty CSR"),
    (lambda c: {**c, "slide": [], "wall_faces": [], "seam_face": [np.zeros(4, np.int32)]}, ValueError, "seam_face"),
])
def test_malformed_topology_wire_is_refused_before_the_device(core, bad, exc, match):
    args, kwargs = _topo_new()
    with pytest.raises(exc, match=match):
        core.CppStructuredSweepSession(*args, **{**kwargs, "control": bad(kwargs["control"])})


def test_batch_refuses_a_topology_wire(core):
    args, kwargs = _topo_new()
    with pytest.raises(NotImplementedError, match="batch"):
        core.CppBatchSweepSession([tuple(args)], dim=kwargs["dim"], control=[kwargs["control"]])


# ---------------------------------------------------------------- GPU ----


def _session(core, name, wire=None, precision="fp64"):
    g, (ctx, st, X) = _session_args(name)
    return g, core.CppStructuredSweepSession(ctx, st, X, dim=g.d, control=wire or _wire(name), precision=precision)


@pytest.mark.gpu
def test_set_c_evaluates_the_net(gpu):
    g, s = _session(gpu, "wavy9")
    w = _wire("wavy9")
    shape = g.blocks[0].shape
    C0 = w["C0"].reshape(5, 5, 2)
    s.set_C(C0.reshape(-1))
    bases = control.axis_bases(shape, (5, 5))
    Xn = control.prolong(bases, C0) + w["b"].reshape(shape + (2,))
    X = s.get_X().reshape(-1, 2)
    np.testing.assert_allclose(X[g.blocks[0].reshape(-1)], Xn.reshape(-1, 2), atol=1e-12)
    np.testing.assert_allclose(s.get_C(), w["C0"], atol=1e-14)


@pytest.mark.gpu
def test_run_control_rejects_untangle_and_needs_a_wire(gpu):
    g, s = _session(gpu, "wavy9")
    with pytest.raises(ValueError, match="untangle"):
        s.run_control(1, phase="untangle")
    plain = gpu.CppStructuredSweepSession(g.wire(), g.structured(), g.X_flat())
    with pytest.raises(ValueError, match="control wire"):
        plain.run_control(1)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CONTROL_CASES))
def test_run_control_matches_reference_core(gpu, name):
    src, kw, ctrl, blk, phase, n_outer, opts, _ = CONTROL_CASES[name]
    g, s = _session(gpu, name)
    rep = s.run_control(n_outer, phase=phase, **opts)
    pre = f"{name}/ref/"
    assert rep["iters"] == int(_FX[pre + "iters"])
    assert bool(rep["converged"]) == bool(_FX[pre + "converged"])
    # near convergence the energy is a sum of round-off (cube9c reaches ~1e-13)
    e_ref = _FX[pre + "energies"]
    np.testing.assert_allclose(rep["energies"], e_ref, rtol=1e-9, atol=1e-12 * abs(e_ref[0]))
    np.testing.assert_allclose(rep["mindets"], _FX[pre + "mindets"], rtol=1e-8)
    np.testing.assert_array_equal(rep["alphas"], _FX[pre + "alphas"])
    assert len(rep["pcg_iters"]) == len(_FX[pre + "pcg_iters"])
    assert np.all(np.abs(np.asarray(rep["pcg_iters"]) - _FX[pre + "pcg_iters"]) <= 1)
    scale = np.abs(g.X).max()
    np.testing.assert_allclose(s.get_X(), _FX[pre + "X"], rtol=0, atol=1e-8 * scale)
    np.testing.assert_allclose(s.get_C(), _FX[pre + "C"], rtol=0, atol=1e-8 * scale)
    assert np.all(np.diff(rep["energies"]) <= 1e-12)


@pytest.mark.gpu
def test_run_control_matches_numpy_dense_oracle(gpu):
    """The reference's own parity bar (tests/smoothing/test_control_cpp.py:105-150)."""
    src, kw, ctrl, blk, phase, n_outer, opts, _ = CONTROL_CASES["wavy13"]
    g, s = _session(gpu, "wavy13")
    rep = s.run_control(n_outer, **opts)
    e_ref = _FX["wavy13/numpy/energies"]
    e = np.asarray(rep["energies"])
    assert np.all(np.isfinite(e)) and np.all(np.asarray(rep["mindets"]) > 0)
    assert abs(rep["iters"] - int(_FX["wavy13/numpy/iters"])) <= 2
    n = min(e.size, e_ref.size)
    np.testing.assert_allclose(e[:n], e_ref[:n], rtol=1e-7)
    np.testing.assert_allclose(s.get_X(), _FX["wavy13/numpy/X"], atol=1e-6)


@pytest.mark.gpu
def test_own_wire_builder_runs_like_the_reference_wire(gpu):
    g, s = _session(gpu, "disk17c")
    w = control.control_wire(control.grid_block_nodes(g, 0), (6, 6), block=0)
    _, s2 = _session(gpu, "disk17c", wire=w)
    r1, r2 = s.run_control(8), s2.run_control(8)
    np.testing.assert_allclose(r2["energies"], r1["energies"], rtol=1e-10)


@pytest.mark.gpu
def test_control_then_nodal_interop(gpu):
    g, s = _session(gpu, "wavy9")
    rep = s.run_control(5)
    E, M = s.run(10, phase="barrier", omega=0.8)
    assert np.isfinite(E[-1]) and M[-1] > 0 and E[-1] <= rep["energies"][-1] + 1e-9


@pytest.mark.gpu
def test_batch_of_nets_equals_separate_sessions(gpu):
    ms = [configs.multiblock_mesh(s, lo=17, hi=49) for s in (40, 41, 42)]
    wires = []
    for g in ms:
        b = int(np.argmax([blk.size for blk in g.blocks]))
        shape = g.blocks[b].shape
        wires.append(control.control_wire(control.grid_block_nodes(g, b), tuple(min(8, n - 2) for n in shape),
                                          block=b))
    bs = gpu.CppBatchSweepSession([(g.wire(compact=True), g.structured(), g.X_flat()) for g in ms], control=wires)
    reps = bs.run_control(6)
    Xb = bs.get_X()
    for m, g in enumerate(ms):
        s = gpu.CppStructuredSweepSession(g.wire(compact=True), g.structured(), g.X_flat(), control=wires[m])
        r = s.run_control(6)
        assert reps[m]["iters"] == r["iters"]
        np.testing.assert_allclose(reps[m]["energies"], r["energies"], rtol=1e-11)
        np.testing.assert_array_equal(reps[m]["alphas"], r["alphas"])
        np.testing.assert_allclose(Xb[m], s.get_X(), atol=1e-12)
