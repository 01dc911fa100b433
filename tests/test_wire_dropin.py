"""wire.build_flat_context as a drop-in for the reference's own
build_flat_context (egg/smoothing/flat_context.py:136-346): same arguments,
same wire.  Runs where the reference's Python package is importable (the
build container); the index arrays come from the host builder here, and
tests/test_wire_gpu.py pins the device arrays to the host builder's, so the
two together cover the device path end to end."""

from __future__ import annotations

import numpy as np
import pytest

from egg_b200 import configs, wire
from oracle import oracle

_ROOT = oracle.reference_root()
pytestmark = pytest.mark.skipif(_ROOT is None, reason="reference checkout absent")


@pytest.fixture
def ref_fc(monkeypatch):
    monkeypatch.syspath_prepend(str(_ROOT))
    fc = pytest.importorskip("egg.smoothing.flat_context")
    monkeypatch.setattr(wire, "_device_arrays",
                        lambda b, m, st, d, syn, ea, dev: wire._host_arrays(b, m, st, d, syn, ea))
    return fc


def _same(a, b, where=""):
    if isinstance(a, dict):
        assert isinstance(b, dict) and set(a) == set(b), (where, sorted(set(a) ^ set(b)))
        for k in a:
            _same(a[k], b[k], f"{where}/{k}")
    elif isinstance(a, (list, tuple)):
        assert len(a) == len(b), where
        for i, (x, y) in enumerate(zip(a, b)):
            _same(x, y, f"{where}[{i}]")
    elif isinstance(a, np.ndarray):
        b = np.asarray(b)
        assert a.dtype == b.dtype and a.shape == b.shape, (where, a.dtype, b.dtype, a.shape, b.shape)
        np.testing.assert_array_equal(a, b, err_msg=where)
    else:
        assert a == b, (where, a, b)


def _both(fc, g, dof_entities, **kw):
    blocks = [np.asarray(b) for b in g.blocks]
    ref = fc.build_flat_context(blocks, g.free, dof_entities, g.d, **kw)
    got = wire.build_flat_context(blocks, g.free, dof_entities, g.d, device="cuda:0", **kw)
    _same(ref, got)


def test_free_dofs_uniform_and_per_sample_targets(ref_fc):
    g = configs.disk_oh(17, frac=0.25, seed=2)
    ns = sum(4 * (b.shape[0] - 1) * (b.shape[1] - 1) for b in g.blocks)
    w = np.eye(2) + 0.1 * np.random.default_rng(0).standard_normal((ns, 2, 2))
    for w_inv in (np.eye(2), 2.0 * np.eye(2), np.array([[1.0, 0.2], [0.0, 1.3]]), w):
        _both(ref_fc, g, {}, w_inv=w_inv)


def test_constrained_dofs_take_the_reference_entity_partitions(ref_fc):
    from egg.geometry.analytic2d import Circle

    g = configs.disk_on_curve(17)
    free = g.free.copy()
    ents = {}
    for n in g.constraints:
        free[n] = True
        ents[n] = Circle((0.0, 0.0), 1.0)
    g.free = free
    _both(ref_fc, g, ents, w_inv=np.eye(2))


def test_soft_term_tables(ref_fc):
    from egg.smoothing.directional import DirectionalSamples
    from egg.smoothing.interface_c2 import CurvatureWindows

    g = configs.with_soft_terms(configs.unit_square(17, frac=0.2, seed=3), seed=1)
    dr, cu = g.soft["directional"], g.soft["curvature"]
    ds = DirectionalSamples(nodes=dr["nodes"], kind=dr["kind"], ref=dr["ref"], axis=dr["axis"], weight=dr["weight"],
                            eps=dr["eps"])
    cw = CurvatureWindows(nodes=cu["nodes"], weight=cu["weight"])
    _both(ref_fc, g, {}, w_inv=np.eye(2), directional=ds, curvature=cw)


def test_3d_sphere_in_cube(ref_fc):
    g = configs.sphere_in_cube(9, seed=1)
    _both(ref_fc, g, {}, w_inv=np.eye(3))


def test_interface_samples_are_refused(ref_fc):
    g = configs.unit_square(9)

    class _Iface:
        def __len__(self):
            return 3

    with pytest.raises(NotImplementedError, match="interface"):
        wire.build_flat_context(g.blocks, g.free, {}, 2, w_inv=np.eye(2), interface=_Iface())
