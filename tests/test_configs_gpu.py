"""Parity at the benchmark configurations' own sizes, against runs of the
reference core (fp64 build) recorded in tests/golden/ref_configs.npz by
tests/golden/gen_golden_fixtures.py --configs:

* C1  disk O-H, 5 blocks of 65^2, +-0.25h, shape, 40 sweeps (exactly the config);
* C3  1025^2 square with ~5% of cells inverted: the delta-continuation untangle
      schedule (egg/smoothing/cpp_backend.py:773-848), then 100 shape+size
      sweeps with the mean-size target;
* C4  7-block sphere-in-cube at 33^3, +-0.2h: untangle, then FAS V(2,2) with
      at most 4 levels;
* C5  32 multi-block meshes (3-9 blocks, sides 17..257) in one batched
      session, 20 sweeps.

fp64 is held to the reference at the tolerances of the small-grid tests
(positions 1e-12 h after one sweep, 1e-9 h over a trajectory; energies 1e-9
relative, FAS cycles 1e-8).  The mixed path is held to the north star's bar:
first-sweep positions within 1e-5 h, the same untangle status and delta-step
count, energies within 1e-6 relative of the fp64 reference.
"""

from __future__ import annotations

import numpy as np
import pytest

from egg_b200 import configs, driver
from tests.conftest import GOLDEN
from tests.golden.gen_golden_fixtures import C3_SHAPE_SIZE_SWEEPS, C4_CYCLES, C5_MESHES, CONFIG_STRIDE

pytestmark = pytest.mark.gpu

_REF = np.load(GOLDEN / "ref_configs.npz")
PRECISIONS = ["fp64", "mixed"]


def _hmin(g):
    return float(configs._min_edge(g.blocks, g.X).min())


def _session(core, g, precision, **kw):
    return core.CppStructuredSweepSession(g.wire(**kw), g.structured(), g.X_flat(), dim=g.d, precision=precision)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_c1_disk_oh65_40_sweeps(gpu, precision):
    g = configs.disk_oh(65, frac=0.25, seed=0)
    h = _hmin(g)
    s = _session(gpu, g, precision)
    e1, _ = s.run(1, report_every=1)
    dx1 = np.abs(s.get_X() - _REF["c1/X1"]).max()
    s = _session(gpu, g, precision)
    E, M = s.run(40, report_every=1)
    dxn = np.abs(s.get_X() - _REF["c1/X40"]).max()
    if precision == "fp64":
        assert dx1 <= 1e-12 * h, dx1 / h
        np.testing.assert_allclose(e1, _REF["c1/E1"], rtol=1e-12)
        np.testing.assert_allclose(E, _REF["c1/E"], rtol=1e-9)
        np.testing.assert_allclose(M, _REF["c1/M"], rtol=1e-8)
        assert dxn <= 1e-9 * h, dxn / h
    else:
        assert dx1 <= 1e-5 * h, dx1 / h
        np.testing.assert_allclose(E[-1], _REF["c1/E"][-1], rtol=1e-6)
    assert np.sign(M[-1]) == np.sign(_REF["c1/M"][-1])


@pytest.mark.parametrize("precision", PRECISIONS)
def test_c3_untangle1025_then_shape_size(gpu, precision):
    g = configs.tangled_square(1025, target=0.05, seed=0)
    h = 1.0 / 1024
    k = CONFIG_STRIDE["c3"]
    md0 = float(configs.grid_mindet(g.blocks, g.X).min())
    np.testing.assert_allclose(md0, float(_REF["c3/mindet0"]), rtol=1e-12)
    a = driver.structured_session(g, compact=True, precision=precision)
    md, outer, _ = driver.untangle(a, sweeps_per_delta=20)
    ref_mds = _REF["c3/untangle_mindets"]
    # untangle status and schedule length match exactly
    assert outer == ref_mds.size
    assert (md > 0) == (ref_mds[-1] > 0)
    Xu = a.get_X()
    b = gpu.CppStructuredSweepSession(g.wire(compact=True, w_inv=configs.mean_size_w_inv(g.blocks, g.X)),
                                      g.structured(), Xu, precision=precision)
    E, M = b.run(C3_SHAPE_SIZE_SWEEPS, phase="shape_size", report_every=10)
    dxu = np.abs(Xu.reshape(-1, 2)[::k] - _REF["c3/Xu"]).max()
    dx = np.abs(b.get_X().reshape(-1, 2)[::k] - _REF["c3/X"]).max()
    if precision == "fp64":
        np.testing.assert_allclose(md, ref_mds[-1], rtol=1e-8)
        assert dxu <= 1e-9 * h, dxu / h
        np.testing.assert_allclose(E, _REF["c3/E"], rtol=1e-9)
        np.testing.assert_allclose(M, _REF["c3/M"], rtol=1e-7)
        assert dx <= 1e-9 * h, dx / h
    else:
        np.testing.assert_allclose(E[-1], _REF["c3/E"][-1], rtol=1e-6)
    assert np.sign(M[-1]) == np.sign(_REF["c3/M"][-1])


@pytest.mark.parametrize("precision", PRECISIONS)
def test_c4_sphere_in_cube33_untangle_fas(gpu, precision):
    g = configs.sphere_in_cube(33, frac=0.2, seed=0)
    s = _session(gpu, g, precision, compact=True)
    md, outer, _ = driver.untangle(s, sweeps_per_delta=20)
    ref_mds = _REF["c4/untangle_mindets"]
    assert outer == ref_mds.size
    if outer:
        assert (md > 0) == (ref_mds[-1] > 0)
    E, M = s.run_fas(C4_CYCLES, nu_pre=2, nu_post=2, max_levels=4)
    levels = np.array([[list(t) for t in lv] for lv in s.mg_levels()], dtype=np.int32).reshape(
        len(s.mg_levels()), -1)
    np.testing.assert_array_equal(levels, _REF["c4/levels"])
    h = _hmin(g)
    dx = np.abs(s.get_X().reshape(-1, 3)[:: CONFIG_STRIDE["c4"]] - _REF["c4/X"]).max()
    if precision == "fp64":
        if outer:
            np.testing.assert_allclose(md, ref_mds[-1], rtol=1e-8)
        np.testing.assert_allclose(E, _REF["c4/E"], rtol=1e-8)
        np.testing.assert_allclose(M, _REF["c4/M"], rtol=1e-6)
        assert dx <= 1e-7 * h, dx / h
    else:
        np.testing.assert_allclose(E, _REF["c4/E"], rtol=1e-6)
    assert np.sign(M[-1]) == np.sign(_REF["c4/M"][-1])


@pytest.mark.parametrize("precision", PRECISIONS)
def test_c5_batch_of_32_meshes(gpu, precision):
    ms = configs.batch_meshes(C5_MESHES, seed=0)
    b = gpu.CppBatchSweepSession([(g.wire(compact=True), g.structured(), g.X_flat()) for g in ms],
                                 precision=precision)
    E, M = b.run(20, report_every=10)
    assert E.shape == _REF["c5/E"].shape
    X = np.concatenate([x.reshape(-1, 2) for x in b.get_X()])[:: CONFIG_STRIDE["c5"]]
    dx = np.abs(X - _REF["c5/X"]).max()
    h = 1.0 / 256
    if precision == "fp64":
        np.testing.assert_allclose(E, _REF["c5/E"], rtol=1e-9)
        np.testing.assert_allclose(M, _REF["c5/M"], rtol=1e-8)
        assert dx <= 1e-9 * h, dx / h
    else:
        np.testing.assert_allclose(E, _REF["c5/E"], rtol=1e-6)
    np.testing.assert_array_equal(np.sign(M[:, -1]), np.sign(_REF["c5/M"][:, -1]))
