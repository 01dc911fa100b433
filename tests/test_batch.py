"""Batched sessions: several independent multi-block meshes in one store.

CPU part: the mesh generator and the host-side merge validation (the merge
runs before any device is touched).  GPU part: a batch sweeps every mesh
exactly as separate sessions do on the same kernel variant (positions
bit-identical, per-mesh energies to rounding), the report chunks replayed from CUDA graphs equal the
launch-by-launch path, and every mesh matches the oracle."""

from __future__ import annotations

import os

import numpy as np
import pytest

from egg_b200 import configs
from oracle import oracle
from tests.conftest import gpu_available


def _meshes(n=5, seed=3, lo=9, hi=33):
    return configs.batch_meshes(n, seed=seed, lo=lo, hi=hi)


def _tuples(ms, compact=True):
    return [(g.wire(compact=compact), g.structured(), g.X_flat()) for g in ms]


# ---------------------------------------------------------------- CPU ----


def test_multiblock_mesh_is_conforming():
    for seed in range(12):
        g = configs.multiblock_mesh(seed, lo=9, hi=33)
        assert 3 <= len(g.blocks) <= 9
        ids = np.concatenate([b.ravel() for b in g.blocks])
        assert ids.min() == 0 and ids.max() == g.num_nodes - 1
        # every node appears in some block, interface nodes in two or more
        cnt = np.bincount(ids, minlength=g.num_nodes)
        assert cnt.min() >= 1 and cnt.max() <= 4
        # fixed nodes are exactly the outline; the interior moves
        assert 0 < g.num_free < g.num_nodes
        h = g.meta["h"]
        edges = configs._min_edge(g.blocks, g.X)
        assert edges.min() > 0.4 * h


def test_batch_meshes_are_seeded():
    a, b = configs.batch_meshes(3, seed=1), configs.batch_meshes(3, seed=1)
    for ga, gb in zip(a, b):
        np.testing.assert_array_equal(ga.X, gb.X)


def test_batch_merge_rejects_out_of_range_indices(core):
    ms = _meshes(3)
    t = _tuples(ms)
    ctx = dict(t[1][0])
    grp = dict(ctx["groups"][0])
    gc = np.array(grp["gc"], dtype=np.int32).copy()
    if gc.size == 0:
        pytest.skip("mesh 1 has no stored samples")
    gc[0] = ms[1].num_nodes  # one past mesh 1's nodes: valid in the merged numbering
    grp["gc"] = gc
    ctx["groups"] = [grp]
    t[1] = (ctx, t[1][1], t[1][2])
    with pytest.raises(ValueError, match="batch mesh 1"):
        core.CppBatchSweepSession(t)


def test_batch_merge_rejects_mixed_energy_stencils(core):
    ms = _meshes(2)
    t = [(ms[0].wire(compact=True), ms[0].structured(), ms[0].X_flat()),
         (ms[1].wire(compact=False), ms[1].structured(), ms[1].X_flat())]
    with pytest.raises(NotImplementedError, match="mix"):
        core.CppBatchSweepSession(t)


@pytest.mark.skipif(gpu_available(), reason="a GPU is present")
def test_batch_without_device_raises(core):
    with pytest.raises(RuntimeError, match="no CUDA device"):
        core.CppBatchSweepSession(_tuples(_meshes(2)))


# ---------------------------------------------------------------- GPU ----


def _hmin(g):
    return float(configs._min_edge(g.blocks, g.X).min())


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_equals_separate_sessions(gpu, precision):
    ms = _meshes(6)
    b = gpu.CppBatchSweepSession(_tuples(ms), precision=precision)
    b.set_variant(1)  # bit-identity holds on the same kernel variant
    assert b.num_meshes == 6
    Eb, Mb = b.run(12, report_every=4)
    assert Eb.shape == (6, 3) and Mb.shape == (6, 3)
    Xb = b.get_X()
    for m, g in enumerate(ms):
        s = gpu.CppStructuredSweepSession(g.wire(compact=True), g.structured(), g.X_flat(), precision=precision)
        s.set_variant(1)
        E, M = s.run(12, report_every=4)
        np.testing.assert_array_equal(Xb[m], s.get_X())
        np.testing.assert_allclose(Eb[m], E, rtol=1e-13)
        np.testing.assert_array_equal(Mb[m], M)
    Ee, Me = b.energy()
    np.testing.assert_allclose(Ee, Eb[:, -1], rtol=1e-13)
    np.testing.assert_array_equal(Me, Mb[:, -1])


@pytest.mark.gpu
def test_batch_matches_oracle_per_mesh(gpu):
    ms = _meshes(4, seed=5)
    for phase, delta, omega in (("barrier", 0.0, 0.9), ("untangle", 1e-3, 0.5), ("shape_size", 0.0, 1.0)):
        b = gpu.CppBatchSweepSession(_tuples(ms, compact=False))
        E, M = b.run(6, phase=phase, delta=delta, omega=omega, report_every=2)
        Xb = b.get_X()
        for m, g in enumerate(ms):
            Xo, Eo, Mo = oracle.run(g.X, oracle.patches_for(g.blocks, g.free), oracle.stencil_for(g.blocks), 6,
                                    phase=phase, delta=delta, omega=omega, report_every=2)
            assert np.abs(Xb[m] - Xo.ravel()).max() <= 1e-11 * _hmin(g)
            np.testing.assert_allclose(E[m], Eo, rtol=1e-11)
            np.testing.assert_allclose(M[m], Mo, rtol=1e-10)


@pytest.mark.gpu
@pytest.mark.parametrize("k", [1, 2, 3, 5])
def test_graph_chunks_equal_direct_launches(gpu, k, monkeypatch):
    g = configs.disk_oh(17, frac=0.25, seed=9)
    runs = {}
    for flag in ("1", "0"):
        monkeypatch.setenv("EGG_B200_GRAPHS", flag)
        s = gpu.CppStructuredSweepSession(g.wire(), g.structured(), g.X_flat())
        s.set_variant(1)
        E, M = s.run(17, report_every=k)
        E2, M2 = s.run(6, report_every=k)
        runs[flag] = (E, M, E2, M2, s.get_X(), s.launch_count())
    for a, b in zip(runs["1"][:5], runs["0"][:5]):
        np.testing.assert_array_equal(a, b)
    assert runs["1"][5] == runs["0"][5]


@pytest.mark.gpu
def test_batch_set_get_roundtrip_and_3d(gpu):
    ms = [configs.unit_cube(7, frac=0.15, seed=1), configs.two_cubes(5, frac=0.15, seed=2),
          configs.unit_cube(9, frac=0.15, seed=3)]
    b = gpu.CppBatchSweepSession(_tuples(ms), dim=3)
    b.set_variant(1)
    X0 = b.get_X()
    for x, g in zip(X0, ms):
        np.testing.assert_array_equal(x, g.X_flat())
    E, M = b.run(8, report_every=4)
    for m, g in enumerate(ms):
        s = gpu.CppStructuredSweepSession(g.wire(compact=True), g.structured(), g.X_flat(), dim=3)
        s.set_variant(1)
        Es, Ms = s.run(8, report_every=4)
        np.testing.assert_array_equal(b.get_X()[m], s.get_X())
        np.testing.assert_allclose(E[m], Es, rtol=1e-13)
    b.set_X(X0)
    E2, _ = b.run(8, report_every=4)
    np.testing.assert_array_equal(E2, E)


@pytest.mark.gpu
def test_batch_refuses_fas(gpu):
    b = gpu.CppBatchSweepSession(_tuples(_meshes(2)))
    with pytest.raises(NotImplementedError, match="batch"):
        b.run_fas(1)
