"""Soft energy terms on the GPU: grids carrying directional samples (parallel,
line, stem; 2D and 3D) and 2D curvature windows relax exactly as the reference
core relaxes them (first sweep and trajectory, fp64, the reported energy being
the composed objective), structured-interior DOFs with terms leave the tile
path, sliding boundary DOFs take the directional samples only, FAS V-cycles
match the reference's, the mixed path tracks fp64, batch sessions relax
each mesh's terms as the reference does, and control nets take the
directional gradient and the composed objective."""

from __future__ import annotations

import numpy as np
import pytest

from egg_b200 import configs
from tests.conftest import GOLDEN
from tests.golden.gen_golden_fixtures import CONTROL_SOFT, FAS_RUNS_SOFT, RUNS_SOFT, case_grid

pytestmark = pytest.mark.gpu

_FX = np.load(GOLDEN / "ref_soft.npz")


def _hmin(g):
    return float(configs._min_edge(g.blocks, g.X).min())


def _session(core, g, precision="fp64", compact=False):
    return core.CppStructuredSweepSession(g.wire(compact=compact), g.structured(), g.X_flat(), dim=g.d,
                                          precision=precision)


@pytest.mark.parametrize("run", RUNS_SOFT, ids=lambda r: f"{r[0]}-{r[1]}-{r[3]}")
def test_soft_sweeps_match_reference(gpu, run):
    case, phase, delta, omega, n = run
    g = case_grid(case)
    key = f"{case}/{phase}/{omega}"
    s = _session(gpu, g)
    s.run(1, phase=phase, delta=delta, omega=omega)
    assert np.abs(s.get_X() - _FX[key + "/X1"]).max() <= 1e-12 * _hmin(g)
    s2 = _session(gpu, g)
    E, M = s2.run(n, phase=phase, delta=delta, omega=omega, report_every=1)
    np.testing.assert_allclose(E, _FX[key + "/E"], rtol=1e-9)
    np.testing.assert_allclose(M, _FX[key + "/M"], rtol=1e-8, atol=1e-16)
    assert np.abs(s2.get_X() - _FX[key + "/Xn"]).max() <= 1e-9 * _hmin(g)


def test_reported_energy_is_the_composed_objective(gpu):
    """The report adds the whole-sample directional total (no curvature), so
    energy() differs from the same grid without terms by exactly that total."""
    g = case_grid("square_soft17")
    with_terms = _session(gpu, g).energy()[0]
    plain = case_grid("square_soft17")
    ds = plain.soft["directional"]
    plain.soft = {}
    base = _session(gpu, plain).energy()[0]
    X = g.X
    tot = 0.0
    for nd, k, r, w in zip(ds["nodes"], ds["kind"], ds["ref"], ds["weight"]):
        eps = ds["eps"]
        if k in (0, 2):
            u = X[nd[1]] - X[nd[0]] if k == 0 else X[nd[0]] - X[nd[1]]
            c = (u @ r) / np.sqrt(u @ u + eps * eps)
            tot += w * c * c
        else:
            q1, q2 = X[nd[0]] - X[nd[1]], X[nd[2]] - X[nd[1]]
            h = q1 / np.sqrt(q1 @ q1 + eps * eps) + q2 / np.sqrt(q2 @ q2 + eps * eps)
            tot += w * (h @ h)
    assert with_terms == pytest.approx(base + tot, rel=1e-12)


@pytest.mark.parametrize("run", FAS_RUNS_SOFT, ids=lambda r: f"{r[0]}-{r[1]}-{r[7]}")
def test_soft_fas_matches_reference(gpu, run):
    """FAS: the fine smoothing and the restricted gradient carry the terms,
    the coarse-correction ladder gates on the composed objective."""
    case, phase, nc, npre, npost, ncoarse, omega, ml = run
    g = case_grid(case)
    key = f"fas/{case}/{phase}/{ml}"
    s = _session(gpu, g)
    E, M = s.run_fas(nc, nu_pre=npre, nu_post=npost, nu_coarse=ncoarse, omega=omega, max_levels=ml, phase=phase)
    np.testing.assert_allclose(E, _FX[key + "/E"], rtol=1e-8)
    np.testing.assert_allclose(M, _FX[key + "/M"], rtol=1e-7, atol=1e-16)
    assert np.abs(s.get_X() - _FX[key + "/X"]).max() <= 1e-8 * _hmin(g)


@pytest.mark.parametrize("case", ["square_soft17", "cube_soft7"])
def test_soft_mixed_tracks_fp64(gpu, case):
    g = case_grid(case)
    key = f"{case}/barrier/1.0"
    n = len(_FX[key + "/E"])
    s = _session(gpu, g, precision="mixed", compact=True)
    s.run(1)
    assert np.abs(s.get_X() - _FX[key + "/X1"]).max() <= 1e-5 * _hmin(g)
    s2 = _session(gpu, g, precision="mixed", compact=True)
    E, M = s2.run(n, report_every=1)
    np.testing.assert_allclose(E[-1], _FX[key + "/E"][-1], rtol=1e-5)
    assert np.sign(M[-1]) == np.sign(_FX[key + "/M"][-1])


def test_soft_batch_matches_reference_per_mesh(gpu):
    """A batch of meshes with different soft-term widths (and one without
    terms) relaxes each mesh as the reference does, and reports each mesh's
    composed objective."""
    plain = case_grid("square_soft17")
    plain.soft = {}
    gs = [case_grid("square_soft17"), case_grid("slide_soft17"), case_grid("disk_oh_soft17"), plain]
    b = gpu.CppBatchSweepSession([(g.wire(), g.structured(), g.X_flat()) for g in gs], precision="fp64")
    E, M = b.run(30, report_every=1)
    Xb = b.get_X()
    for m, case in enumerate(["square_soft17", "slide_soft17", "disk_oh_soft17"]):
        key = f"{case}/barrier/1.0"
        np.testing.assert_allclose(E[m], _FX[key + "/E"], rtol=1e-9)
        np.testing.assert_allclose(M[m], _FX[key + "/M"], rtol=1e-8, atol=1e-16)
        assert np.abs(Xb[m] - _FX[key + "/Xn"]).max() <= 1e-9 * _hmin(gs[m])
    s = _session(gpu, plain)
    Ep, _ = s.run(30, report_every=1)
    np.testing.assert_allclose(E[3], Ep, rtol=1e-12)
    Ee, _ = b.energy()
    np.testing.assert_allclose(Ee, E[:, -1], rtol=1e-12)
    g3 = [case_grid("cube_soft7"), configs.unit_cube(5, seed=3)]
    b3 = gpu.CppBatchSweepSession([(g.wire(), g.structured(), g.X_flat()) for g in g3], dim=3, precision="fp64")
    E3, _ = b3.run(15, report_every=1)
    np.testing.assert_allclose(E3[0], _FX["cube_soft7/barrier/1.0/E"], rtol=1e-9)


@pytest.mark.parametrize("case, blk, ctrl, n_outer", CONTROL_SOFT, ids=lambda v: str(v))
def test_soft_control_net_matches_reference(gpu, case, blk, ctrl, n_outer):
    """A control net on a grid with soft terms: the reduced gradient takes
    the directional samples' nodal gradient, every accept energy the
    composed objective (the net's block holds the terms in both cases)."""
    g = case_grid(case)
    pre = f"control/{case}/"
    w = {k[len(pre + "wire/"):]: _FX[k] for k in _FX.files if k.startswith(pre + "wire/")}
    w["block"] = int(w["block"])
    w["k_supp"] = int(w["k_supp"])
    s = gpu.CppStructuredSweepSession(g.wire(), g.structured(), g.X_flat(), dim=g.d, control=w)
    rep = s.run_control(n_outer)
    assert rep["iters"] == int(_FX[pre + "iters"])
    e_ref = _FX[pre + "energies"]
    np.testing.assert_allclose(rep["energies"], e_ref, rtol=1e-9, atol=1e-12 * abs(e_ref[0]))
    np.testing.assert_allclose(rep["mindets"], _FX[pre + "mindets"], rtol=1e-8)
    np.testing.assert_array_equal(rep["alphas"], _FX[pre + "alphas"])
    scale = np.abs(g.X).max()
    np.testing.assert_allclose(s.get_X(), _FX[pre + "X"], rtol=0, atol=1e-8 * scale)
    np.testing.assert_allclose(s.get_C(), _FX[pre + "C"], rtol=0, atol=1e-8 * scale)


def test_soft_batch_of_control_nets_matches_reference(gpu):
    """Two soft-term meshes with one net each, solved together: each mesh's
    reduced gradient takes only its own directional samples."""
    cases = [c for c, *_ in CONTROL_SOFT]
    gs = [case_grid(c) for c in cases]
    wires = []
    for c in cases:
        pre = f"control/{c}/wire/"
        w = {k[len(pre):]: _FX[k] for k in _FX.files if k.startswith(pre)}
        w["block"] = int(w["block"])
        w["k_supp"] = int(w["k_supp"])
        wires.append(w)
    bs = gpu.CppBatchSweepSession([(g.wire(compact=True), g.structured(), g.X_flat()) for g in gs], control=wires)
    reps = bs.run_control(CONTROL_SOFT[0][3])
    Xb = bs.get_X()
    for m, (c, g) in enumerate(zip(cases, gs)):
        pre = f"control/{c}/"
        assert reps[m]["iters"] == int(_FX[pre + "iters"])
        e_ref = _FX[pre + "energies"]
        np.testing.assert_allclose(reps[m]["energies"], e_ref, rtol=1e-9, atol=1e-12 * abs(e_ref[0]))
        np.testing.assert_allclose(Xb[m], _FX[pre + "X"], rtol=0, atol=1e-8 * np.abs(g.X).max())
