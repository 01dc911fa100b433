"""FAS V-cycles on the GPU against the reference core's own run_fas
(recorded per-cycle energies, final positions, hierarchy shapes) and the
properties the reference tests check (tests/smoothing/test_fas.py)."""

from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from egg_b200 import configs
from tests.conftest import GOLDEN
from tests.golden.gen_golden_fixtures import FAS_RUNS, case_grid

pytestmark = pytest.mark.gpu

_REF = np.load(GOLDEN / "ref_sweeps.npz")


def _hmin(g):
    return float(configs._min_edge(g.blocks, g.X).min())


def _session(core, g, precision="fp64"):
    return core.CppStructuredSweepSession(g.wire(), g.structured(), g.X_flat(), dim=g.d, precision=precision)


@pytest.mark.parametrize("run", FAS_RUNS, ids=lambda r: f"{r[0]}-{r[1]}-L{r[7]}")
def test_fas_hierarchy_matches_reference(gpu, run):
    case, phase, nc, npre, npost, ncoarse, omega, ml = run
    g = case_grid(case)
    s = _session(gpu, g)
    got = np.array([[list(t) for t in lv] for lv in s.mg_levels()], dtype=np.int32).reshape(-1)
    np.testing.assert_array_equal(got, _REF[f"fp64/fas/{case}/{phase}/{ml}/levels"].reshape(-1))


@pytest.mark.parametrize("run", FAS_RUNS, ids=lambda r: f"{r[0]}-{r[1]}-L{r[7]}")
def test_fas_fp64_matches_reference(gpu, run):
    case, phase, nc, npre, npost, ncoarse, omega, ml = run
    g = case_grid(case)
    key = f"fp64/fas/{case}/{phase}/{ml}"
    s = _session(gpu, g)
    E, M = s.run_fas(nc, nu_pre=npre, nu_post=npost, nu_coarse=ncoarse, omega=omega, max_levels=ml, phase=phase)
    e_ref = _REF[key + "/E"]
    # near the minimiser the energy is a sum of round-off: floor at 1e-12 of E0
    np.testing.assert_allclose(E, e_ref, rtol=1e-8, atol=1e-12 * abs(e_ref[0]))
    np.testing.assert_allclose(M, _REF[key + "/M"], rtol=1e-7, atol=1e-16)
    assert np.abs(s.get_X() - _REF[key + "/X"]).max() <= 1e-8 * _hmin(g)


@pytest.mark.parametrize("run", FAS_RUNS, ids=lambda r: f"{r[0]}-{r[1]}-L{r[7]}")
def test_fas_mixed_tracks_reference(gpu, run):
    case, phase, nc, npre, npost, ncoarse, omega, ml = run
    g = case_grid(case)
    key = f"fp64/fas/{case}/{phase}/{ml}"
    s = _session(gpu, g, precision="mixed")
    E, M = s.run_fas(nc, nu_pre=npre, nu_post=npost, nu_coarse=ncoarse, omega=omega, max_levels=ml, phase=phase)
    e64, e32 = _REF[key + "/E"][-1], _REF[f"fp32/fas/{case}/{phase}/{ml}/E"][-1]
    assert abs(E[-1] - e64) <= max(1e-6 * abs(e64), 2.0 * abs(e32 - e64)), (E[-1], e64, e32)
    assert np.sign(M[-1]) == np.sign(_REF[key + "/M"][-1])


def _bump_square(n=17, size=4.0, amp=0.08):
    """Single block of side `size` with a smooth low-frequency displacement
    that vanishes on the boundary, the error plain Jacobi damps slowest
    (reference tests/smoothing/test_fas.py:38-63)."""
    g = configs.unit_square(n, frac=0.0)
    X = g.X * size
    s = np.sin(np.pi * X / size)
    bump = s[:, 0] * s[:, 1]
    X[:, 0] += amp * bump
    X[:, 1] += 0.7 * amp * bump
    return dataclasses.replace(g, X=X, name=f"bump{n}")


def test_fas_levels_of_a_17_node_block(gpu):
    s = _session(gpu, _bump_square())
    assert s.mg_levels() == [[(9, 9)], [(5, 5)], [(3, 3)]]


def test_fas_monotone_and_barrier(gpu):
    """Per-cycle energies non-increasing, min det positive every cycle
    (reference tests/smoothing/test_fas.py:81-91)."""
    s = _session(gpu, _bump_square())
    E, M = s.run_fas(6, omega=0.8)
    assert E.shape == (6,) and np.all(np.isfinite(E)) and np.all(M > 0.0)
    assert np.all(E[1:] <= E[:-1] + 1e-10 * np.maximum(1.0, np.abs(E[:-1])))


def test_fas_beats_jacobi_at_equal_fine_budget(gpu):
    """5 V(2,2) cycles land below half of 20 plain Jacobi sweeps
    (reference tests/smoothing/test_fas.py:94-110)."""
    g = _bump_square()
    Ef, _ = _session(gpu, g).run_fas(5, nu_pre=2, nu_post=2, omega=0.8)
    Ej, _ = _session(gpu, g).run(5 * 2 * 2, omega=0.8)
    assert Ef[-1] <= 0.5 * Ej[-1] + 1e-9, (Ef[-1], Ej[-1])


def test_fas_falls_back_to_jacobi_without_levels(gpu):
    g = case_grid("square33")
    a = _session(gpu, g)
    a.set_variant(1)  # the same kernel variant on both sides
    Ea, Ma = a.run_fas(3, nu_pre=2, nu_post=2, max_levels=1)
    b = _session(gpu, g)
    b.set_variant(1)
    Eb, Mb = b.run(12, report_every=4)
    np.testing.assert_array_equal(Ea, Eb)


def test_fas_rejects_untangle(gpu):
    g = case_grid("square33")
    s = _session(gpu, g)
    with pytest.raises(ValueError, match="untangle"):
        s.run_fas(1, phase="untangle")


def test_fas_agrees_with_jacobi_minimiser(gpu):
    """Long FAS reaches the energy of long Jacobi (same minimiser, different
    path; reference tests/smoothing/test_fas.py:113-125)."""
    g = _bump_square()
    Ef, _ = _session(gpu, g).run_fas(12, omega=0.8)
    Ej, _ = _session(gpu, g).run(600, omega=0.8)
    assert Ef[-1] <= Ej[-1] + 1e-8 * max(1.0, abs(Ej[-1])), (Ef[-1], Ej[-1])



@pytest.mark.parametrize("make,prec", [(lambda: configs.unit_square(257, frac=0.3, seed=2), "mixed"),
                                       (lambda: configs.sphere_in_cube(17, frac=0.15, seed=1), "fp64")],
                         ids=["square257-mixed", "sphere17-fp64"])
def test_fas_coarse_levels_tuned_per_level(gpu, make, prec):
    """Coarse levels pick their own tile variant on their first smoothing;
    the V-cycles then match a session whose variant is pinned on every level
    up to the rounding of the kernel variants, and pinned sessions repeat
    bit for bit."""
    g = make()
    a = _session(gpu, g, prec)
    Ea, Ma = a.run_fas(3, nu_pre=2, nu_post=2, max_levels=4)
    v = a.variants()["variant"]
    runs = []
    for _ in range(2):
        b = _session(gpu, g, prec)
        b.set_variant(v)
        runs.append(b.run_fas(3, nu_pre=2, nu_post=2, max_levels=4))
    np.testing.assert_array_equal(runs[0][0], runs[1][0])
    np.testing.assert_array_equal(runs[0][1], runs[1][1])
    tol = 1e-9 if prec == "fp64" else 1e-6  # fp32 coarse tiles round differently per variant
    np.testing.assert_allclose(Ea, runs[0][0], rtol=tol)
    np.testing.assert_allclose(Ma, runs[0][1], rtol=1e3 * tol)
    Ea2, _ = a.run_fas(1, nu_pre=2, nu_post=2, max_levels=4)  # tuned levels are kept across calls
    assert np.isfinite(Ea2).all() and Ea2[0] <= Ea[-1] + 1e-9 * abs(Ea[-1])
