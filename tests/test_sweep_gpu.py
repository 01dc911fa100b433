"""Parity of the CUDA sweep with the reference (recorded runs + golden
vectors) and with the CPU oracle.  Tolerances: first-sweep positions within
1e-12 h (fp64) / 1e-5 h (mixed), h = the smallest edge of the initial grid."""

from __future__ import annotations

import json

import numpy as np
import pytest

from egg_b200 import configs, driver
from oracle import oracle
from tests.conftest import GOLDEN
from tests.golden.gen_golden_fixtures import RUNS, case_grid

pytestmark = pytest.mark.gpu

_REF = np.load(GOLDEN / "ref_sweeps.npz")


def _hmin(g):
    return float(configs._min_edge(g.blocks, g.X).min())


def _session(core, g, precision="fp64", **kw):
    return core.CppStructuredSweepSession(g.wire(**kw), g.structured(), g.X_flat(), precision=precision)


def test_metric_eval_matches_golden(gpu):
    for r in json.loads((GOLDEN / "golden_metric.json").read_text())["records"]:
        mu, g, H = gpu.metric_eval(np.array(r["t"]))
        np.testing.assert_allclose(mu, r["mu"], rtol=1e-13, atol=1e-14)
        np.testing.assert_allclose(g, r["grad"], rtol=1e-12, atol=1e-13)
        np.testing.assert_allclose(H, r["hess"], rtol=1e-12, atol=1e-12)


def test_metric_eval_shape_size_and_untangle_match_oracle(gpu):
    rng = np.random.default_rng(3)
    for _ in range(16):
        t = rng.normal(size=4) + np.array([1.0, 0.0, 0.0, 1.0])
        for name, kind, delta in (("shape_size", "shape_size", 0.0), ("untangle", "untangle", 0.2)):
            mu, g, H = gpu.metric_eval(t, name, delta)
            mo, go, Ho = oracle.metric(t, kind, delta)
            np.testing.assert_allclose(mu, mo, rtol=1e-13, atol=1e-13)
            np.testing.assert_allclose(g, go, rtol=1e-12, atol=1e-12)
            np.testing.assert_allclose(H, Ho, rtol=1e-11, atol=1e-11)


def test_patch_eval_matches_golden(gpu):
    for r in json.loads((GOLDEN / "golden_patch.json").read_text())["records"]:
        P, n = int(r["P"]), int(r["n_nodes"])
        g, h, e, md = gpu.patch_eval(
            np.array(r["X"][: 2 * n]), np.array(r["gc"][:P]), np.array(r["gn0"][:P]), np.array(r["gn1"][:P]),
            np.array(r["s0"][:P]), np.array(r["s1"][:P]), np.array(r["W_inv"][: 4 * P]), np.array(r["role"][:P]),
            None)
        np.testing.assert_allclose(g, r["grad"], rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(h, r["hess"], rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(e, r["energy"], rtol=1e-13, atol=1e-14)
        np.testing.assert_allclose(md, r["mindet"], rtol=1e-13, atol=1e-14)
        if int(r["tag"]) == 0:
            st = gpu.newton_step(np.array(r["grad"]), np.array(r["hess"]), np.zeros(2), 0, None)
            np.testing.assert_allclose(st, r["delta"], rtol=1e-12, atol=1e-13)


@pytest.mark.parametrize("run", RUNS, ids=lambda r: f"{r[0]}-{r[1]}-{r[3]}")
def test_first_sweep_fp64_matches_reference(gpu, run):
    case, phase, delta, omega, n = run
    g = case_grid(case)
    key = f"fp64/{case}/{phase}/{omega}"
    s = _session(gpu, g)
    e1, m1 = s.run(1, phase=phase, delta=delta, omega=omega, report_every=1)
    dx = np.abs(s.get_X() - _REF[key + "/X1"]).max()
    assert dx <= 1e-12 * _hmin(g), dx
    np.testing.assert_allclose(e1, _REF[key + "/E1"], rtol=1e-12)


@pytest.mark.parametrize("run", RUNS, ids=lambda r: f"{r[0]}-{r[1]}-{r[3]}")
def test_trajectory_fp64_matches_reference(gpu, run):
    case, phase, delta, omega, n = run
    g = case_grid(case)
    key = f"fp64/{case}/{phase}/{omega}"
    s = _session(gpu, g)
    E, M = s.run(n, phase=phase, delta=delta, omega=omega, report_every=1)
    np.testing.assert_allclose(E, _REF[key + "/E"], rtol=1e-9)
    np.testing.assert_allclose(M, _REF[key + "/M"], rtol=1e-8, atol=1e-16)
    assert np.abs(s.get_X() - _REF[key + "/Xn"]).max() <= 1e-9 * _hmin(g)
    assert np.sign(M[-1]) == np.sign(_REF[key + "/M"][-1])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", ["disk_oh33", "square65"])
def test_every_launch_variant_matches_reference(gpu, case, precision):
    """Each interior-kernel variant (cell tiles and full-DOF tiles, whose
    edges fall on different nodes of these 33- and 65-node blocks) relaxes
    the first sweep and the trajectory as the reference does."""
    phase, omega, n = "barrier", 0.8, 40
    g = case_grid(case)
    key = f"fp64/{case}/{phase}/{omega}"
    t1 = 1e-12 if precision == "fp64" else 1e-5
    nv = len(_session(gpu, g).variants()["table"])
    for v in range(nv):
        s = _session(gpu, g, precision=precision)
        s.set_variant(v)
        s.run(1, phase=phase, omega=omega)
        dx = np.abs(s.get_X() - _REF[key + "/X1"]).max()
        assert dx <= t1 * _hmin(g), (v, dx / _hmin(g))
        E, M = s.run(n - 1, phase=phase, omega=omega, report_every=n - 1)
        np.testing.assert_allclose(E[-1], _REF[key + "/E"][-1], rtol=1e-9 if precision == "fp64" else 1e-4)
        assert np.sign(M[-1]) == np.sign(_REF[key + "/M"][-1])


@pytest.mark.parametrize("run", RUNS, ids=lambda r: f"{r[0]}-{r[1]}-{r[3]}")
def test_first_sweep_mixed_within_1e5_h(gpu, run):
    case, phase, delta, omega, n = run
    g = case_grid(case)
    key = f"fp64/{case}/{phase}/{omega}"
    s = _session(gpu, g, precision="mixed")
    s.run(1, phase=phase, delta=delta, omega=omega)
    dx = np.abs(s.get_X() - _REF[key + "/X1"]).max()
    assert dx <= 1e-5 * _hmin(g), dx / _hmin(g)
    E, M = s.run(n - 1, phase=phase, delta=delta, omega=omega, report_every=1)
    np.testing.assert_allclose(E[-1], _REF[key + "/E"][-1], rtol=1e-4)
    assert np.sign(M[-1]) == np.sign(_REF[key + "/M"][-1])


@pytest.mark.parametrize("case", ["square65", "disk_oh33"])
def test_fp64_matches_oracle_on_the_fly(gpu, case):
    g = case_grid(case)
    for phase, delta, omega in (("barrier", 0.0, 0.9), ("shape_size", 0.0, 1.0), ("untangle", 1e-3, 0.5)):
        s = _session(gpu, g)
        E, M = s.run(6, phase=phase, delta=delta, omega=omega, report_every=2)
        Xo, Eo, Mo = oracle.run(g.X, oracle.patches_for(g.blocks, g.free), oracle.stencil_for(g.blocks), 6,
                                phase=phase, delta=delta, omega=omega, report_every=2)
        assert np.abs(s.get_X() - Xo.ravel()).max() <= 1e-11 * _hmin(g)
        np.testing.assert_allclose(E, Eo, rtol=1e-11)
        np.testing.assert_allclose(M, Mo, rtol=1e-10)


def test_mean_size_target_keeps_identity_interior_quirk(gpu):
    """shape_size with W = hbar I: interior DOFs relax with W_inv = I (reference
    src/structured_patch.hpp:183-185); the reported energy uses the true W."""
    g = configs.unit_square(33, frac=0.3, seed=9)
    w = configs.mean_size_w_inv(g.blocks, g.X)
    s = _session(gpu, g, w_inv=w)
    E, M = s.run(5, phase="shape_size", report_every=1)
    Xo, Eo, Mo = oracle.run(g.X, oracle.patches_for(g.blocks, g.free, w), oracle.stencil_for(g.blocks, w), 5,
                            phase="shape_size", report_every=1)
    assert np.abs(s.get_X() - Xo.ravel()).max() <= 1e-11 * _hmin(g)
    np.testing.assert_allclose(E, Eo, rtol=1e-11)


def test_uniform_grid_is_the_minimiser(gpu):
    """Known answer (reference tests/smoothing/test_structured_sweep.py:159-174)."""
    g = configs.unit_square(9, frac=0.0)
    uniform = g.X.copy()
    rng = np.random.default_rng(42)
    X0 = uniform.copy()
    X0[g.free] += rng.normal(0, 0.02, size=(g.num_free, 2))
    s = gpu.CppStructuredSweepSession(g.wire(), g.structured(), X0.ravel())
    _e, m = s.run(3000)
    assert m[-1] > 0
    np.testing.assert_allclose(s.get_X(), uniform.ravel(), atol=1e-9)


def test_report_cadence_and_energy_probe(gpu):
    g = case_grid("square33")
    s = _session(gpu, g)
    e, m = s.run(10, report_every=0)
    assert e.shape == (1,)
    e3, m3 = s.run(10, report_every=3)
    assert e3.shape == (4,)
    e_now, m_now = s.energy()
    assert e_now == pytest.approx(e3[-1], rel=1e-14) and m_now == m3[-1]
    assert s.run(0)[0].shape == (0,)


def test_set_get_roundtrip_and_restart(gpu):
    g = case_grid("disk_oh17")
    s = _session(gpu, g)
    s.set_variant(1)  # the same kernel variant as s2 below
    np.testing.assert_array_equal(s.get_X(), g.X_flat())
    s.run(5)
    s.set_X(g.X_flat())
    np.testing.assert_array_equal(s.get_X(), g.X_flat())
    e_a, _ = s.run(3, report_every=1)
    s2 = _session(gpu, g)
    s2.set_variant(1)
    e_b, _ = s2.run(3, report_every=1)
    np.testing.assert_array_equal(e_a, e_b)


def test_set_get_remap_copies_unblocked_nodes_and_slices(gpu):
    """get_X/set_X remap between global node order and the packed store on the device.

    Every copy of a node shared by blocks takes the value set, nodes in no block
    return their last value set and sweeps leave them alone, and grids large
    enough for several host copy slices round-trip bit for bit (2D and 3D).
    """
    g = case_grid("disk_oh17")
    extra = np.array([0.9, 0.9, -0.9, 0.9, 0.1, -0.95])  # three nodes in no block
    X = np.concatenate([g.X_flat(), extra])
    s = gpu.CppStructuredSweepSession(g.wire(), g.structured(), X, precision="fp64")
    s.set_variant(1)  # the same kernel variant as s2 below
    np.testing.assert_array_equal(s.get_X(), X)
    s.run(5)
    np.testing.assert_array_equal(s.get_X()[-6:], extra)
    rng = np.random.default_rng(3)
    Xr = X + 1e-3 * rng.standard_normal(X.shape)
    s.set_X(Xr)
    np.testing.assert_array_equal(s.get_X(), Xr)
    # every copy took the value: the next sweep equals a fresh session's
    s.set_X(X)
    e_a, _ = s.run(2, report_every=1)
    s2 = gpu.CppStructuredSweepSession(g.wire(), g.structured(), X, precision="fp64")
    s2.set_variant(1)
    e_b, _ = s2.run(2, report_every=1)
    np.testing.assert_array_equal(e_a, e_b)
    np.testing.assert_array_equal(s.get_X(), s2.get_X())
    for big in (configs.unit_square(1025, seed=4), configs.unit_cube(65, seed=4)):
        b = gpu.CppStructuredSweepSession(big.wire(), big.structured(), big.X_flat(), dim=big.d, precision="mixed")
        Xb = big.X_flat() + 1e-4 * rng.standard_normal(big.X_flat().shape)
        b.set_X(Xb)
        np.testing.assert_array_equal(b.get_X(), Xb)
        b.run(1)
        assert not np.array_equal(b.get_X(), Xb)
        b.set_X(Xb)
        np.testing.assert_array_equal(b.get_X(), Xb)


def test_untangle_schedule_clears_folds_like_the_oracle(gpu):
    g = configs.tangled_square(33, seed=4)
    s = _session(gpu, g)
    md, outer, delta = driver.untangle(s)
    assert md > 1e-9 and outer >= 1
    # oracle: same schedule on the CPU restatement
    pt, sc = oracle.patches_for(g.blocks, g.free), oracle.stencil_for(g.blocks)
    X = g.X.copy()
    _, md0 = oracle.energy(X, sc)
    dl = 2.0 * max(abs(md0), 1e-12)
    for it in range(60):
        X, _, M = oracle.run(X, pt, sc, 20, phase="untangle", delta=dl, omega=0.5)
        if M[-1] > 1e-9:
            break
        dl *= 0.8
    assert it + 1 == outer
    assert np.abs(s.get_X() - X.ravel()).max() <= 1e-9 * _hmin(g)


def test_large_grid_properties(gpu):
    """1025^2: monotone energy in both precisions; on a valid (+-0.25h) grid
    the mixed trajectory tracks fp64; on a +-0.3h grid with inverted samples
    (ill-conditioned, where even the reference's own fp32 build departs from
    its fp64 build by percents) the untangle status still matches."""
    for frac, seed in ((0.25, 11), (0.3, 11)):
        g = configs.unit_square(1025, frac=frac, seed=seed)
        E, M = {}, {}
        for prec in ("fp64", "mixed"):
            s = _session(gpu, g, precision=prec, compact=True)
            E[prec], M[prec] = s.run(30, report_every=1)
            assert np.all(np.diff(E[prec]) <= 1e-9 * abs(E[prec][0]))
        assert np.sign(M["mixed"][-1]) == np.sign(M["fp64"][-1])
        if frac == 0.25:
            assert M["fp64"][-1] > 0
            np.testing.assert_allclose(E["mixed"], E["fp64"], rtol=1e-6)


@pytest.mark.parametrize("run", RUNS, ids=lambda r: f"{r[0]}-{r[1]}-{r[3]}")
def test_mixed_trajectory_tracks_fp64_reference(gpu, run):
    """After 40 sweeps the mixed sweep's energy is within 1e-6 relative of the
    fp64 reference (or within twice the reference's own fp32 build deviation,
    whichever is larger) and has the same min-det sign.  Positions are held to
    2e-3 h: near a minimum fp32 patch energies (absolute noise ~1e-6, the
    reference fp32 line-search slack) only locate the minimiser to about
    sqrt(eps_f) h ~ 3e-4 h."""
    case, phase, delta, omega, n = run
    g = case_grid(case)
    s = _session(gpu, g, precision="mixed")
    E, M = s.run(n, phase=phase, delta=delta, omega=omega, report_every=1)
    key64, key32 = f"fp64/{case}/{phase}/{omega}", f"fp32/{case}/{phase}/{omega}"
    e64, e32 = _REF[key64 + "/E"][-1], _REF[key32 + "/E"][-1]
    tol = max(1e-6 * abs(e64), 2.0 * abs(e32 - e64))
    assert abs(E[-1] - e64) <= tol, (E[-1], e64, e32)
    assert np.abs(s.get_X() - _REF[key64 + "/Xn"]).max() <= 2e-3 * _hmin(g)
    assert np.sign(M[-1]) == np.sign(_REF[key64 + "/M"][-1])


def test_mixed_shape_size_on_small_cells_tracks_fp64(gpu):
    """With the identity target the size term makes mu ~ 1 on small cells and
    a Newton step changes it by ~1e-12, below what fp32 resolves of mu itself;
    the mixed line search accepts on exact metric differences and so tracks
    the fp64 sweep (untangle, then shape+size with the mean-size target)."""
    g = configs.tangled_square(257, target=0.05, seed=3)
    w = configs.mean_size_w_inv(g.blocks, g.X)
    res = {}
    for prec in ("fp64", "mixed"):
        a = driver.structured_session(g, compact=True, precision=prec)
        md, _outer, _delta = driver.untangle(a)
        assert md > 0
        b = gpu.CppStructuredSweepSession(g.wire(compact=True, w_inv=w), g.structured(), a.get_X(),
                                          precision=prec)
        E, M = b.run(300, phase="shape_size", report_every=100)
        assert M[-1] > 0
        res[prec] = E
    assert abs(res["mixed"][-1] - res["fp64"][-1]) <= 1e-3 * abs(res["fp64"][-1])


def test_singular_owner_override_changes_nothing(gpu):
    """sing_block / sing_logical pick which block's copy of a fan node the core
    treats as its owner (the reference's singular-node host choice); the sweep
    is the same whichever block owns it."""
    g = case_grid("disk_oh17")
    st = g.structured()
    ids0 = g.blocks[0]
    sb, sl = [], []
    for gid in (ids0[0, 0], ids0[0, -1], ids0[-1, 0], ids0[-1, -1]):  # valence-3 nodes
        for b in range(len(g.blocks) - 1, 0, -1):  # the highest block holding the node
            hit = np.argwhere(g.blocks[b] == gid)
            if hit.size:
                sb.append(b)
                sl.append(hit[0])
                break
    assert len(sb) == 4
    st2 = dict(st, sing_block=np.asarray(sb, dtype=np.int32), sing_logical=np.asarray(sl, dtype=np.int32))
    a = gpu.CppStructuredSweepSession(g.wire(), st, g.X_flat())
    b = gpu.CppStructuredSweepSession(g.wire(), st2, g.X_flat())
    a.set_variant(1)
    b.set_variant(1)
    Ea, Ma = a.run(6, report_every=2)
    Eb, Mb = b.run(6, report_every=2)
    np.testing.assert_array_equal(a.get_X(), b.get_X())
    np.testing.assert_allclose(Ea, Eb, rtol=1e-14)


def test_get_x_results_are_independent_pooled_arrays(gpu):
    """get_X hands out page-locked pooled buffers: every result is its own
    array (no aliasing between live results), and a buffer recycled after its
    array is freed carries the new positions."""
    g = case_grid("square33")
    s = _session(gpu, g)
    a = s.get_X()
    s.run(2)
    b = s.get_X()
    assert not np.shares_memory(a, b)
    np.testing.assert_array_equal(a, g.X_flat())
    b_copy = b.copy()
    a[:] = -1.0
    np.testing.assert_array_equal(b, b_copy)
    del a
    s.run(1)
    c = s.get_X()
    assert not np.shares_memory(b, c)
    assert not np.array_equal(c, b_copy)
    s.set_X(c)
    np.testing.assert_array_equal(s.get_X(), c)


def test_set_X_from_page_locked_and_pageable_buffers(gpu):
    """set_X takes one DMA from a page-locked array (a get_X result comes from
    the core's pinned pool) and threaded staging from pageable memory; both
    land the same positions, and a later sweep starts from them."""
    g = configs.disk_oh(17, frac=0.25, seed=2)
    s = gpu.CppStructuredSweepSession(g.wire(), g.structured(), g.X_flat(), device="cuda:0")
    s.run(3)
    Xp = s.get_X()
    Xq = np.array(Xp, copy=True)
    t = gpu.CppStructuredSweepSession(g.wire(), g.structured(), g.X_flat(), device="cuda:0")
    t.set_X(Xp)
    np.testing.assert_array_equal(t.get_X(), Xq)
    Ea, _ = t.run(2, report_every=1)
    t.set_X(Xq)
    np.testing.assert_array_equal(t.get_X(), Xq)
    Eb, _ = t.run(2, report_every=1)
    np.testing.assert_array_equal(Ea, Eb)
