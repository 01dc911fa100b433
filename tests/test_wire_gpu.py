"""The device-side wire build (egg_b200_wire_build) equals the host builder
and the reference's build_flat_context output, bit for bit."""

from __future__ import annotations

import numpy as np
import pytest

from egg_b200 import configs, wire
from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _same(a, b, where=""):
    """Recursive exact equality of two wire dicts (values, dtypes, shapes)."""
    if isinstance(a, dict):
        assert isinstance(b, dict) and set(a) == set(b), (where, sorted(set(a) ^ set(b)))
        for k in a:
            _same(a[k], b[k], f"{where}/{k}")
    elif isinstance(a, list):
        assert isinstance(b, list) and len(a) == len(b), where
        for i, (x, y) in enumerate(zip(a, b)):
            _same(x, y, f"{where}[{i}]")
    elif isinstance(a, np.ndarray):
        b = np.asarray(b)
        assert a.dtype == b.dtype and a.shape == b.shape, (where, a.dtype, b.dtype, a.shape, b.shape)
        np.testing.assert_array_equal(a, b, err_msg=where)
    else:
        assert a == b and type(a) is type(b), (where, a, b)


def _grids():
    yield configs.disk_oh(17, frac=0.25, seed=2)
    yield configs.unit_square(33)
    yield configs.two_squares(17, 6)
    yield configs.multiblock_mesh(3, lo=9, hi=33)
    yield configs.unit_cube(9)
    yield configs.sphere_in_cube(9, seed=1)
    yield configs.square_sliding(17)
    yield configs.disk_on_curve(17)
    yield configs.square_bspline(17)
    yield configs.cube_bsurf(9)
    yield configs.with_soft_terms(configs.unit_square(17, frac=0.2, seed=3), seed=1)


@pytest.mark.parametrize("g", list(_grids()), ids=lambda g: g.name)
def test_device_wire_equals_host_wire(gpu, g):
    for compact in (False, True):
        _same(g.wire(compact=compact), g.wire(compact=compact, device="cuda:0"))


def test_device_wire_non_uniform_targets(gpu):
    """Per-sample W_inv rows gather through the device's per-row sample ids;
    an anisotropic uniform target keeps every DOF on a stored patch."""
    g = configs.disk_oh(17, frac=0.25, seed=2)
    ns = sum(4 * (b.shape[0] - 1) * (b.shape[1] - 1) for b in g.blocks)
    rng = np.random.default_rng(0)
    w = np.eye(2) + 0.1 * rng.standard_normal((ns, 2, 2))
    for w_inv in (w, np.array([[1.0, 0.2], [0.0, 1.3]])):
        _same(g.wire(w_inv=w_inv), g.wire(w_inv=w_inv, device="cuda:0"))


def test_device_wire_matches_reference_builder(gpu):
    ref = np.load(GOLDEN / "ref_wire_disk_oh17.npz")
    g = configs.disk_oh(17, frac=0.25, seed=2)
    for tag, w in (("eye", np.eye(2)), ("aniso", np.array([[1.0, 0.2], [0.0, 1.3]]))):
        ctx = wire.flat_wire(g.blocks, g.free, 2, w_inv=w, device="cuda:0")
        for part, key in (("group", ctx["groups"][0]), ("es", ctx["energy_stencil"])):
            for k, v in key.items():
                if isinstance(v, np.ndarray):
                    np.testing.assert_array_equal(v.reshape(-1), ref[f"{tag}/{part}/{k}"].reshape(-1), k)


def test_device_wire_session_runs_like_host_wire(gpu):
    g = configs.disk_oh(17, frac=0.25, seed=2)
    core = gpu
    out = []
    for dev in (None, "cuda:0"):
        s = core.CppStructuredSweepSession(g.wire(device=dev), g.structured(), g.X_flat(), device="cuda:0")
        s.set_variant(0)  # one kernel variant on both sides (variants agree only to rounding)
        E, M = s.run(4, report_every=2)
        out.append((s.get_X(), E, M))
    for a, b in zip(out[0], out[1]):
        np.testing.assert_array_equal(a, b)


def test_device_wire_large_grid(gpu):
    """1025^2 with a released boundary rail (stored DOFs on every face): the
    counting sort by node and the energy stencil at size."""
    g = configs.unit_square(1025, frac=0.3, seed=4)
    free = g.free.copy()
    edge = np.concatenate([g.blocks[0][0, 1:-1], g.blocks[0][-1, 1:-1]])
    free[edge] = True
    a = wire.flat_wire(g.blocks, free, 2)
    b = wire.flat_wire(g.blocks, free, 2, device="cuda:0")
    _same(a, b)
    assert a["groups"][0]["P_of"].sum() == a["groups"][0]["gc"].size > 0


def test_device_wire_edge_cases(gpu):
    core = gpu
    # a block without cells (one node wide) and an empty moving set
    blocks = [np.arange(12).reshape(3, 4), np.arange(12, 16).reshape(1, 4)]
    free = np.zeros(16, dtype=bool)
    _same(wire.flat_wire(blocks, free, 2), wire.flat_wire(blocks, free, 2, device="cuda:0"))
    free[[5, 6, 13]] = True
    _same(wire.flat_wire(blocks, free, 2), wire.flat_wire(blocks, free, 2, device="cuda:0"))
    # ids outside [0, num_nodes) are refused
    with pytest.raises(ValueError, match="out of range"):
        core.wire_build(2, np.array([3, 4], dtype=np.int32), np.arange(12, dtype=np.int64) + 5,
                        np.zeros(12, dtype=np.uint8))
    with pytest.raises(ValueError, match="block_ids length"):
        core.wire_build(2, np.array([3, 4], dtype=np.int32), np.arange(11, dtype=np.int64),
                        np.zeros(12, dtype=np.uint8))


@pytest.mark.parametrize("make", [lambda: configs.unit_square(513, frac=0.3, seed=1),
                                  lambda: configs.disk_oh(65, frac=0.25, seed=0)], ids=["square513", "disk_oh65"])
def test_reference_form_wire_sessions(gpu, make):
    """A reference-form wire (per-sample energy-stencil arrays, checked and
    remapped on host threads) gives the compact wire's sweeps bit for bit;
    with its samples permuted (no longer the canonical stencil) it takes
    the stored-stencil reduction, whose energies agree to rounding."""
    g = make()
    full, comp = g.wire(device="cuda:0"), g.wire(compact=True, device="cuda:0")
    es = full["energy_stencil"]
    perm = np.random.default_rng(0).permutation(es["num_samples"])
    shuffled = {**full, "energy_stencil": {**es, **{k: es[k][perm] for k in es
                                                   if k[:2] in ("gc", "gn", "s0", "s1")}}}
    out = []
    for ctx in (comp, full, shuffled):
        s = gpu.CppStructuredSweepSession(ctx, g.structured(), g.X_flat(), device="cuda:0")
        s.set_variant(0)  # one kernel variant on every side (variants agree only to rounding)
        E, M = s.run(3, report_every=1)
        out.append((s.get_X(), E, M, s.info()))
    for a, b in zip(out[0][:3], out[1][:3]):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(out[0][0], out[2][0])
    np.testing.assert_allclose(out[2][1], out[0][1], rtol=1e-12)
    np.testing.assert_array_equal(out[2][2], out[0][2])
