"""3D parity of the CUDA sweep (mu_cond3 and its shape_size / untangle
variants, 64-occurrence patches) with the reference and the oracle."""

from __future__ import annotations

import json

import numpy as np
import pytest

from egg_b200 import configs
from oracle import oracle
from tests.conftest import GOLDEN
from tests.golden.gen_golden_fixtures import RUNS3, case_grid

pytestmark = pytest.mark.gpu

_REF = np.load(GOLDEN / "ref_sweeps.npz")


def _hmin(g):
    return float(configs._min_edge(g.blocks, g.X).min())


def _session(core, g, precision="fp64", **kw):
    return core.CppStructuredSweepSession(g.wire(**kw), g.structured(), g.X_flat(), dim=3, precision=precision)


def test_metric3_matches_golden(gpu):
    rng = np.random.default_rng(0)
    for r in json.loads((GOLDEN / "golden_metric_3d.json").read_text())["records"]:
        H = np.array(r["hess"]).reshape(9, 9)
        for _ in range(3):
            v = rng.normal(size=3)
            mu, g9, hv = gpu.metric_eval_3d(np.array(r["t"]), v)
            np.testing.assert_allclose(mu, r["mu"], rtol=1e-12, atol=1e-13)
            np.testing.assert_allclose(g9, r["grad"], rtol=1e-11, atol=1e-12)
            Hb = np.array([[v @ H[3 * i:3 * i + 3, 3 * j:3 * j + 3] @ v for j in range(3)] for i in range(3)])
            ref = Hb[np.triu_indices(3)]
            np.testing.assert_allclose(hv, ref, rtol=1e-10, atol=1e-10 * (1 + np.abs(ref).max()))


def test_metric3_variants_match_oracle(gpu):
    rng = np.random.default_rng(1)
    for name, delta in (("shape_size", 0.0), ("untangle", 0.25)):
        for _ in range(10):
            t = rng.normal(size=9) + 2 * np.eye(3).ravel()
            v = rng.normal(size=3)
            mu, g9, hv = gpu.metric_eval_3d(t, v, name, delta)
            mo, go, Ho = oracle.metric3(t, name, delta)
            Ho = Ho.reshape(9, 9)
            Hb = np.array([[v @ Ho[3 * i:3 * i + 3, 3 * j:3 * j + 3] @ v for j in range(3)] for i in range(3)])
            np.testing.assert_allclose(mu, mo, rtol=1e-12, atol=1e-12)
            np.testing.assert_allclose(g9, go, rtol=1e-11, atol=1e-11)
            np.testing.assert_allclose(hv, Hb[np.triu_indices(3)], rtol=1e-9, atol=1e-9)


@pytest.mark.parametrize("run", RUNS3, ids=lambda r: f"{r[0]}-{r[1]}-{r[3]}")
def test_first_sweep3_fp64_matches_reference(gpu, run):
    case, phase, delta, omega, n = run
    g = case_grid(case)
    key = f"fp64/{case}/{phase}/{omega}"
    s = _session(gpu, g)
    e1, _ = s.run(1, phase=phase, delta=delta, omega=omega, report_every=1)
    dx = np.abs(s.get_X() - _REF[key + "/X1"]).max()
    assert dx <= 1e-12 * _hmin(g), dx
    np.testing.assert_allclose(e1, _REF[key + "/E1"], rtol=1e-12)
    E, M = s.run(n - 1, phase=phase, delta=delta, omega=omega, report_every=1)
    np.testing.assert_allclose(E, _REF[key + "/E"][1:], rtol=1e-9)
    np.testing.assert_allclose(M, _REF[key + "/M"][1:], rtol=1e-8, atol=1e-16)


@pytest.mark.parametrize("run", RUNS3, ids=lambda r: f"{r[0]}-{r[1]}-{r[3]}")
def test_first_sweep3_mixed_within_1e5_h(gpu, run):
    case, phase, delta, omega, n = run
    g = case_grid(case)
    key = f"fp64/{case}/{phase}/{omega}"
    s = _session(gpu, g, precision="mixed")
    s.run(1, phase=phase, delta=delta, omega=omega)
    dx = np.abs(s.get_X() - _REF[key + "/X1"]).max()
    assert dx <= 1e-5 * _hmin(g), dx / _hmin(g)
    E, M = s.run(n - 1, phase=phase, delta=delta, omega=omega, report_every=1)
    e64, e32 = _REF[key + "/E"][-1], _REF[f"fp32/{case}/{phase}/{omega}/E"][-1]
    assert abs(E[-1] - e64) <= max(1e-6 * abs(e64), 2.0 * abs(e32 - e64))
    assert np.sign(M[-1]) == np.sign(_REF[key + "/M"][-1])


def test_fp64_matches_oracle_sphere_in_cube(gpu):
    g = configs.sphere_in_cube(9, frac=0.1, seed=8)
    for phase, delta, omega in (("barrier", 0.0, 0.9), ("untangle", 1e-4, 0.5)):
        s = _session(gpu, g)
        E, M = s.run(3, phase=phase, delta=delta, omega=omega, report_every=1)
        Xo, Eo, Mo = oracle.run3(g.X, oracle.patches_for(g.blocks, g.free, d=3),
                                 oracle.stencil_for(g.blocks, d=3), 3, phase=phase, delta=delta, omega=omega,
                                 report_every=1)
        assert np.abs(s.get_X() - Xo.ravel()).max() <= 1e-10 * _hmin(g)
        np.testing.assert_allclose(E, Eo, rtol=1e-10)


def test_compact_wire_3d_matches_full(gpu):
    g = case_grid("sphere_in_cube7")
    a = _session(gpu, g)
    b = _session(gpu, g, compact=True)
    assert b.info()["structured_energy"] == 1 and a.info()["structured_energy"] == 1
    ea, _ = a.run(4, report_every=1)
    eb, _ = b.run(4, report_every=1)
    np.testing.assert_allclose(ea, eb, rtol=1e-13)
