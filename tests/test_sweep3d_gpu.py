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


def _sample_quality3(ids, X):
    """Per cell and corner sample: det of its edge matrix and det^2 over the
    product of its column norms squared (the kernels' shape test)."""
    n0, n1, n2 = ids.shape
    D = np.zeros((n0 - 1, n1 - 1, n2 - 1, 8))
    Q = np.zeros_like(D)
    for b in range(8):
        o = ((b >> 2) & 1, (b >> 1) & 1, b & 1)
        pc = X[ids[o[0]:o[0] + n0 - 1, o[1]:o[1] + n1 - 1, o[2]:o[2] + n2 - 1]]
        cols = []
        for ax in range(3):
            nb = b ^ (4 >> ax)
            q = ((nb >> 2) & 1, (nb >> 1) & 1, nb & 1)
            s = -1.0 if b & (4 >> ax) else 1.0
            cols.append(s * (X[ids[q[0]:q[0] + n0 - 1, q[1]:q[1] + n1 - 1, q[2]:q[2] + n2 - 1]] - pc))
        T = np.stack(cols, axis=-1)
        D[..., b] = np.linalg.det(T)
        Q[..., b] = D[..., b] ** 2 / np.prod((T * T).sum(axis=-2), axis=-1)
    return D, Q


@pytest.mark.parametrize("phase,delta", [("barrier", 0.0), ("untangle", 1e-4)])
def test_mixed_3d_bad_cell_dofs_relax_in_fp64(gpu, phase, delta):
    """A 17^3 cube with +-0.3h noise holds 86 inverted or badly shaped
    samples.  A DOF whose 8 cells hold one relaxes in fp64 (the tile's
    per-cell masks send it there), so in every mixed kernel variant the DOFs
    next to a clearly bad sample land exactly where the fp64 session puts
    them; the variants agree with one another to rounding (the per-DOF code
    is shared, only the tiling differs); and the whole first sweep stays
    within 5e-5 h of fp64 on this tangled grid (the clean grids hold 1e-5 h)."""
    g = configs.unit_cube(17, frac=0.3, seed=3)
    ids = np.asarray(g.blocks[0])
    D, Q = _sample_quality3(ids, g.X)
    thr2 = 0.1 ** 2
    clearly_bad = ((D <= 0.0) | (Q < 0.5 * thr2)).any(axis=-1)  # per cell
    cb = np.zeros(ids.shape, dtype=bool)  # DOFs (interior nodes) touching such a cell
    for o in np.ndindex(2, 2, 2):
        cb[o[0]:o[0] + 16, o[1]:o[1] + 16, o[2]:o[2] + 16] |= clearly_bad
    cb[0, :, :] = cb[-1, :, :] = cb[:, 0, :] = cb[:, -1, :] = cb[:, :, 0] = cb[:, :, -1] = False
    nodes = ids[cb]
    assert nodes.size > 20
    h = _hmin(g)
    first = None
    for variant in range(5):
        f = _session(gpu, g)
        f.set_variant(variant)
        f.run(1, phase=phase, delta=delta, omega=0.8)
        Xf = f.get_X().reshape(-1, 3)
        m = _session(gpu, g, precision="mixed")
        m.set_variant(variant)
        m.run(1, phase=phase, delta=delta, omega=0.8)
        Xm = m.get_X().reshape(-1, 3)
        # fp64 on both sides (the fp32 path would differ by ~1e-7 h or more)
        np.testing.assert_allclose(Xm[nodes], Xf[nodes], rtol=0, atol=1e-10 * h)
        assert np.abs(Xm - Xf).max() <= 5e-5 * h
        if first is None:
            first = Xm
        else:  # same per-DOF code; instances may contract FMAs differently
            np.testing.assert_allclose(Xm, first, rtol=0, atol=1e-12 * h)
