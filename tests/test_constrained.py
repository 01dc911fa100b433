"""Constrained boundary DOFs (nodes that slide on a 2D curve), CPU part: the
wire's entity partitions, the entity geometry compiled for the host against
the reference core's Newton step and projection, and the host-side
rejections (unsupported tags, malformed records) that run before any device
is touched."""

from __future__ import annotations

import shutil
import subprocess

import numpy as np
import pytest

from egg_b200 import configs
from tests.conftest import GOLDEN, ROOT

_FX = np.load(GOLDEN / "ref_constrained.npz")


@pytest.mark.parametrize("grid", [configs.disk_on_curve(9), configs.disk_on_curve(9, ry=0.6),
                                  configs.disk_on_curve(9, arcs=True), configs.disk_on_curve(9, ry=0.6, arcs=True),
                                  configs.square_sliding(9), configs.square_bezier(9),
                                  configs.cube_sliding(5), configs.cube_curved(5), configs.square_bspline(9),
                                  configs.square_composite(9), configs.square_composite_bspline(9)],
                         ids=lambda g: g.name)
def test_wire_partitions_cover_every_dof_once(grid):
    grp = grid.wire()["groups"][0]
    seen = np.zeros(grp["D"], dtype=int)
    for name, part in grp["entities"].items():
        dl = np.asarray(part["dof_local"])
        seen[dl] += 1
        assert len(part["records"]) == len(dl) * part["kFields"]
        gids = np.asarray(grp["dof_idx"])[dl]
        if part["tag"] == 0:
            assert grid.free[gids].all()
        else:
            assert all(grid.constraints[int(v)][0] == part["tag"] for v in gids)
            assert (np.asarray(grp["interior_block"])[dl] == -1).all()
    assert (seen == 1).all()
    assert grp["D"] == grid.num_free + len(grid.constraints)


def test_entity_geometry_matches_the_reference_core(tmp_path):
    """Newton step reduced onto the tangent (a released rail: the full step;
    zero gradient: no step; a singular reduced system: the -0.1 g/|g|
    fallback) and the projection, for LineSeg, Circle, Ellipse, LineRail and
    the trimmed curves CircleArc, EllipseArc, QuadBezier, CubicBezier (cold:
    the foot re-represented nearest the trim, then clamped)."""
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no host C++ compiler")
    exe = tmp_path / "entity"
    subprocess.run([gxx, "-O1", "-std=c++17", f"-I{ROOT / 'egg_b200' / 'csrc'}", f"-I{ROOT / 'include'}",
                    str(ROOT / "tests" / "native" / "entity_check.cpp"), "-o", str(exe)], check=True)
    for tag in (1, 2, 3, 6, 7, 8, 9, 15):
        k = f"entity/{tag}/"
        rec = np.zeros(10)
        rec[: len(_FX[k + "params"])] = _FX[k + "params"]
        lines = []
        for i in range(len(_FX[k + "pos"])):
            vals = [tag, *rec, *_FX[k + "grad"][i], *_FX[k + "hess"][i], *_FX[k + "pos"][i]]
            lines.append(" ".join(repr(float(v)) if j else str(v) for j, v in enumerate(vals)))
        out = subprocess.run([str(exe)], input="\n".join(lines) + "\n", capture_output=True, text=True,
                             check=True).stdout
        got = np.array([[float(x) for x in ln.split()] for ln in out.strip().split("\n")])
        np.testing.assert_allclose(got[:, :2], _FX[k + "step"], rtol=1e-12, atol=1e-15)
        np.testing.assert_allclose(got[:, 2:], _FX[k + "foot"], rtol=1e-12, atol=1e-15)


def test_entity3_projection_matches_the_reference_core(tmp_path):
    """Sphere, Plane, Cylinder, Line3 (foot, trim clamp, evaluation) and
    LineRail3 (released beyond its ends) projections against the reference's
    batched projection."""
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no host C++ compiler")
    exe = tmp_path / "entity3"
    subprocess.run([gxx, "-O1", "-std=c++17", f"-I{ROOT / 'egg_b200' / 'csrc'}", f"-I{ROOT / 'include'}",
                    str(ROOT / "tests" / "native" / "entity3_check.cpp"), "-o", str(exe)], check=True)
    for tag in (4, 5, 12, 13, 16):
        k = f"entity3/{tag}/"
        rec = np.zeros(10)
        rec[: len(_FX[k + "params"])] = _FX[k + "params"]
        lines = [" ".join([str(tag), *(repr(float(v)) for v in rec), *(repr(float(v)) for v in q)])
                 for q in _FX[k + "pos"]]
        out = subprocess.run([str(exe)], input="\n".join(lines) + "\n", capture_output=True, text=True,
                             check=True).stdout
        got = np.array([[float(x) for x in ln.split()] for ln in out.strip().split("\n")])
        np.testing.assert_allclose(got, _FX[k + "foot"], rtol=1e-12, atol=1e-15)


def _square():
    g = configs.square_sliding(9)
    return g, g.wire(), g.structured(), g.X_flat()


def _with_part(ctx, name, part):
    grp = dict(ctx["groups"][0])
    ents = dict(grp["entities"])
    ents[name] = {**ents[name], **part}
    grp["entities"] = ents
    return {**ctx, "groups": [grp]}


def test_unsupported_entity_tag_is_rejected(core):
    g, ctx, st, X = _square()
    part = ctx["groups"][0]["entities"]["line_seg"]
    n = len(part["dof_local"])
    ctx4 = _with_part(ctx, "line_seg", {"tag": 4, "kFields": 10, "records": np.zeros(10 * n)})  # Sphere
    with pytest.raises(NotImplementedError, match="tag 4"):
        core.CppStructuredSweepSession(ctx4, st, X)


def test_malformed_entity_records_are_rejected(core):
    g, ctx, st, X = _square()
    part = ctx["groups"][0]["entities"]["line_seg"]
    bad = _with_part(ctx, "line_seg", {"records": np.asarray(part["records"])[:-1]})
    with pytest.raises(ValueError, match="records size"):
        core.CppStructuredSweepSession(bad, st, X)
    rec = np.asarray(part["records"]).copy()
    rec[2] = np.nan
    with pytest.raises(ValueError, match="not finite"):
        core.CppStructuredSweepSession(_with_part(ctx, "line_seg", {"records": rec}), st, X)


def test_constrained_interior_dof_is_rejected(core):
    g = configs.unit_square(9, frac=0.1, seed=1)
    ctx, st, X = g.wire(), g.structured(), g.X_flat()
    grp = ctx["groups"][0]
    k = int(np.flatnonzero(np.asarray(grp["interior_block"]) >= 0)[0])
    free = np.setdiff1d(grp["entities"]["free"]["dof_local"], [k]).astype(np.int32)
    ents = {"free": {**grp["entities"]["free"], "dof_local": free},
            "line_seg": {"tag": 1, "kFields": 4, "dof_local": np.array([k], dtype=np.int32),
                         "records": np.array([0.0, 0.0, 1.0, 1.0])}}
    with pytest.raises(NotImplementedError, match="structured-interior"):
        core.CppStructuredSweepSession({**ctx, "groups": [{**grp, "entities": ents}]}, st, X)
