"""The CPU oracle pinned against the reference: its golden vectors, recorded
runs of the reference core, and (when built here) the reference core itself."""

from __future__ import annotations

import json

import numpy as np
import pytest

from oracle import oracle
from tests.conftest import GOLDEN
from tests.golden.gen_golden_fixtures import RUNS, case_grid


def _records(name):
    return json.loads((GOLDEN / f"{name}.json").read_text())["records"]


@pytest.mark.parametrize("rec", _records("golden_metric"), ids=lambda r: str(r["t"][:2]))
def test_metric_matches_reference_golden(rec):
    mu, g, H = oracle.metric(np.array(rec["t"]), "shape")
    np.testing.assert_allclose(mu, rec["mu"], rtol=1e-13, atol=1e-14)
    np.testing.assert_allclose(g, rec["grad"], rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(H, rec["hess"], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("i", range(5))
def test_patch_matches_reference_golden(i):
    r = _records("golden_patch")[i]
    P = int(r["P"])
    n = int(r["n_nodes"])
    X = np.array(r["X"][: 2 * n])
    g, h, e, md, st = oracle.patch(
        X, np.array(r["gc"][:P]), np.array(r["gn0"][:P]), np.array(r["gn1"][:P]), np.array(r["s0"][:P]),
        np.array(r["s1"][:P]), np.array(r["W_inv"][: 4 * P]), np.array(r["role"][:P]))
    np.testing.assert_allclose(g, r["grad"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(h, r["hess"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(e, r["energy"], rtol=1e-13, atol=1e-14)
    np.testing.assert_allclose(md, r["mindet"], rtol=1e-13, atol=1e-14)
    if int(r["tag"]) == 0:  # Free DOF: plain 2x2 Newton step
        np.testing.assert_allclose(st, r["delta"], rtol=1e-12, atol=1e-13)


def test_untangle_closed_form_matches_finite_differences():
    rng = np.random.default_rng(0)
    for _ in range(20):
        t = rng.normal(size=4)
        delta = 0.3
        mu, g, H = oracle.metric(t, "untangle", delta)
        eps = 1e-6
        for k in range(4):
            tp, tm = t.copy(), t.copy()
            tp[k] += eps
            tm[k] -= eps
            mp, gp, _ = oracle.metric(tp, "untangle", delta)
            mm, gm, _ = oracle.metric(tm, "untangle", delta)
            assert abs((mp - mm) / (2 * eps) - g[k]) < 1e-6 * (1 + abs(g[k]))
            np.testing.assert_allclose((gp - gm) / (2 * eps), H[4 * k : 4 * k + 4], rtol=1e-5, atol=1e-5)


_REF = np.load(GOLDEN / "ref_sweeps.npz")


@pytest.mark.parametrize("run", RUNS, ids=lambda r: f"{r[0]}-{r[1]}-{r[3]}")
def test_oracle_matches_recorded_reference(run):
    case, phase, delta, omega, n = run
    g = case_grid(case)
    pt = oracle.patches_for(g.blocks, g.free)
    sc = oracle.stencil_for(g.blocks)
    key = f"fp64/{case}/{phase}/{omega}"
    X1, _, _ = oracle.run(g.X, pt, sc, 1, phase=phase, delta=delta, omega=omega, report_every=1)
    h = 1.0 / (max(b.shape[0] for b in g.blocks) - 1)
    assert np.abs(X1.ravel() - _REF[key + "/X1"]).max() <= 1e-12 * h
    Xn, E, M = oracle.run(g.X, pt, sc, n, phase=phase, delta=delta, omega=omega, report_every=1)
    np.testing.assert_allclose(E, _REF[key + "/E"], rtol=1e-10)
    np.testing.assert_allclose(M, _REF[key + "/M"], rtol=1e-9, atol=1e-15)


def test_oracle_matches_reference_build_when_present():
    ref = oracle.load_ref("fp64")
    if ref is None:
        pytest.skip("oracle/_ref not built in this environment")
    g = case_grid("disk_oh17")
    X, E, M = ref.cpp_structured_sweep(g.wire(), g.structured(), g.X_flat(), 7, device="cpu", omega=0.8,
                                       report_every=2)
    Xo, Eo, Mo = oracle.run(g.X, oracle.patches_for(g.blocks, g.free), oracle.stencil_for(g.blocks), 7,
                            omega=0.8, report_every=2)
    assert np.abs(Xo.ravel() - X).max() < 1e-14
    np.testing.assert_allclose(Eo, E, rtol=1e-13)
    np.testing.assert_allclose(Mo, M, rtol=1e-13)


from tests.golden.gen_golden_fixtures import RUNS3  # noqa: E402


@pytest.mark.parametrize("rec", _records("golden_metric_3d"), ids=lambda r: str(r["t"][:2]))
def test_metric3_matches_reference_golden(rec):
    mu, g, H = oracle.metric3(np.array(rec["t"]), "shape")
    np.testing.assert_allclose(mu, rec["mu"], rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(g, rec["grad"], rtol=1e-11, atol=1e-12)
    np.testing.assert_allclose(H, rec["hess"], rtol=1e-11, atol=1e-11 * (1 + np.abs(rec["hess"]).max()))


@pytest.mark.parametrize("run", RUNS3, ids=lambda r: f"{r[0]}-{r[1]}-{r[3]}")
def test_oracle3_matches_recorded_reference(run):
    case, phase, delta, omega, n = run
    g = case_grid(case)
    pt = oracle.patches_for(g.blocks, g.free, d=3)
    sc = oracle.stencil_for(g.blocks, d=3)
    key = f"fp64/{case}/{phase}/{omega}"
    h = float(__import__("egg_b200.configs", fromlist=["x"])._min_edge(g.blocks, g.X).min())
    X1, _, _ = oracle.run3(g.X, pt, sc, 1, phase=phase, delta=delta, omega=omega, report_every=1)
    assert np.abs(X1.ravel() - _REF[key + "/X1"]).max() <= 1e-12 * h
    Xn, E, M = oracle.run3(g.X, pt, sc, n, phase=phase, delta=delta, omega=omega, report_every=1)
    np.testing.assert_allclose(E, _REF[key + "/E"], rtol=1e-10)
    np.testing.assert_allclose(M, _REF[key + "/M"], rtol=1e-9, atol=1e-15)


def _ref_sweep_energy(build: str, threads: int) -> float:
    """Energy after two sweeps of the recorded O-grid call, by one reference
    build in a fresh process (one cpp_core per process)."""
    import os
    import subprocess
    import sys

    code = (
        "import gzip,pickle,sys; sys.path.insert(0, %r); from oracle import oracle;"
        "ev=[e for e in pickle.load(gzip.open(%r))['events'] if e.get('name')=='cpp_structured_sweep'][0];"
        "ctx,st,X=ev['args'][:3]; kw=dict(ev['kwargs']); kw.update(device='cpu', report_every=2);"
        "print(repr(float(oracle.load_ref(%r).cpp_structured_sweep(ctx,st,X,2,**kw)[1][-1])))"
        % (str(oracle.HERE.parent), str(oracle.HERE.parent / "tests" / "golden" / "ref_dropin.pkl.gz"), build))
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    out = subprocess.run([sys.executable, "-c", code], check=True, capture_output=True, text=True, env=env).stdout
    return float(out.strip().splitlines()[-1])


def test_reference_halo_launch_order_matters_and_the_snapshot_build_is_fixed():
    """On the reference's 12-block O-grid the order inside its fused
    ghost-fill + shared-node-refresh launch changes the result: the serial
    forward order (one OpenMP thread: ghost fills first, from non-owner copies
    not yet refreshed) differs from the snapshot order (refreshes first),
    which is the same for any thread count.  With several threads the OpenMP
    build's result varies from run to run between the two."""
    if not (oracle.ref_path("fp64").exists() and oracle.ref_path("fp64snap").exists()):
        pytest.skip("oracle/_ref not built in this environment")
    e1 = _ref_sweep_energy("fp64", 1)
    s1, s8 = _ref_sweep_energy("fp64snap", 1), _ref_sweep_energy("fp64snap", 8)
    assert s1 == s8
    assert abs(s1 - e1) > 1e-7 * abs(s1)  # 7e-7 here; equivalent orderings agree to ~1e-15
