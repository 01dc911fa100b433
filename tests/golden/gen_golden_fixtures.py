"""Generate the committed golden fixtures under tests/golden/.

Two sources, both from the reference checkout (run in a container that has it):

1. The reference's own golden vectors, read as data from its C++ test headers
   ``tests/cpp/golden_metric.hpp``, ``golden_metric_3d.hpp`` and
   ``golden_patch.hpp`` (written by the reference's ``tests/cpp/gen_golden.py``
   from its C++ oracle bindings) -> ``golden_metric.json``,
   ``golden_metric_3d.json``, ``golden_patch.json``.
2. Runs of the reference core itself, built from source by
   ``oracle/build_ref.sh`` into ``oracle/_ref``, on small seeded grids from
   ``egg_b200.configs`` -> ``ref_sweeps.npz`` (first-sweep positions and
   energy / min-det trajectories), so the GPU tests can compare against the
   reference without the reference present.

3. Constrained boundary runs of the same core (``ref_constrained.npz``):
   sweeps with nodes sliding on Circle, Ellipse, LineSeg and LineRail
   entities, and the entity Newton step / projection on random inputs.

4. Control-net runs of the same reference core and of the reference's NumPy
   dense reduced-GN oracle (``egg.smoothing.control_ref``), with the control
   wires built by the reference's own builders -> ``ref_control.npz``.

5. Soft-term runs of the same core (``ref_soft.npz``): sweeps and FAS cycles
   on grids carrying directional samples and curvature windows, and the
   reference's own soft-term wire tables for the same terms.

Usage: python tests/golden/gen_golden_fixtures.py [REFERENCE_ROOT]
"""

from __future__ import annotations

import json
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

_NUM = r"[+-]?(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?"


def _ref_root() -> Path:
    """The reference checkout to read (``$EGG_REFERENCE_ROOT`` or a sibling
    ``reference/`` of this repository); the script needs it."""
    from oracle import oracle

    root = oracle.reference_root()
    if root is None:
        raise SystemExit("reference checkout not found: pass its path or set EGG_REFERENCE_ROOT")
    return root


def _blocks(text: str) -> list[str]:
    """Top-level ``{ ... }`` records of the kSamples initializer."""
    start = text.index("= {{") + 4
    out, depth, cur = [], 0, []
    for ch in text[start:]:
        if ch == "{":
            depth += 1
            if depth == 1:
                cur = []
                continue
        elif ch == "}":
            if depth == 0:
                break
            depth -= 1
            if depth == 0:
                out.append("".join(cur))
                continue
        if depth >= 1:
            cur.append(ch)
    return out


def _fields(rec: str) -> dict:
    out = {}
    for m in re.finditer(r"\.(\w+)\s*=\s*(\{[^}]*\}|[^,\n]+)", rec):
        key, val = m.group(1), m.group(2).strip()
        nums = [float(x) for x in re.findall(_NUM, val)]
        out[key] = nums if val.startswith("{") else nums[0]
    return out


def parse_header(path: Path) -> list[dict]:
    return [_fields(r) for r in _blocks(path.read_text())]


def gen_reference_vectors(ref_root: Path) -> None:
    cpp = ref_root / "tests" / "cpp"
    for name in ("golden_metric", "golden_metric_3d", "golden_patch"):
        recs = parse_header(cpp / f"{name}.hpp")
        (HERE / f"{name}.json").write_text(
            json.dumps({"source": f"tests/cpp/{name}.hpp", "records": recs}, indent=1)
        )
        print(f"{name}: {len(recs)} records")


# Small seeded cases shared with tests/test_sweep_gpu.py.
CASES = {
    "square33": ("unit_square", dict(n=33, frac=0.3, seed=1), None),
    "square65": ("unit_square", dict(n=65, frac=0.3, seed=7), None),
    "disk_oh17": ("disk_oh", dict(n=17, frac=0.25, seed=2), None),
    "disk_oh33": ("disk_oh", dict(n=33, frac=0.25, seed=5), None),
    "tangled33": ("tangled_square", dict(n=33, seed=4), None),
    "cube9": ("unit_cube", dict(n=9, frac=0.2, seed=3), None),
    "two_cubes7": ("two_cubes", dict(n=7, frac=0.2, seed=4), None),
    "sphere_in_cube7": ("sphere_in_cube", dict(n=7, frac=0.1, seed=5), None),
    "square65s": ("unit_square", dict(n=65, frac=0.25, seed=12), None),
    "disk_oh33s": ("disk_oh", dict(n=33, frac=0.2, seed=13), None),
    "cube17": ("unit_cube", dict(n=17, frac=0.15, seed=14), None),
    "sphere_in_cube9": ("sphere_in_cube", dict(n=9, frac=0.1, seed=15), None),
    "square33f": ("unit_square", dict(n=33, frac=0.2, seed=22), None),
    "two_squares": ("two_squares", dict(n_big=17, n_small=6, frac=0.2, seed=23), None),
}
RUNS = [
    # (case, phase, delta, omega, n_sweeps)
    ("square33", "barrier", 0.0, 1.0, 40),
    ("square65", "barrier", 0.0, 0.8, 40),
    ("disk_oh17", "barrier", 0.0, 1.0, 40),
    ("disk_oh33", "barrier", 0.0, 0.8, 40),
    ("square33", "shape_size", 0.0, 1.0, 40),
    ("tangled33", "untangle", 2e-4, 0.5, 40),
]
# FAS V-cycles: (case, phase, n_cycles, nu_pre, nu_post, nu_coarse, omega, max_levels)
FAS_RUNS = [
    ("square65s", "barrier", 4, 2, 2, 32, 1.0, 32),
    ("square65s", "shape_size", 3, 2, 2, 32, 0.8, 3),
    ("disk_oh33s", "barrier", 4, 2, 2, 32, 0.8, 32),
    ("cube17", "barrier", 3, 2, 2, 32, 1.0, 32),
    ("sphere_in_cube9", "barrier", 3, 2, 2, 16, 0.8, 4),
    ("square33f", "barrier", 40, 2, 2, 32, 1.0, 32),
    ("two_squares", "barrier", 6, 2, 2, 32, 0.8, 32),
]
RUNS3 = [
    ("cube9", "barrier", 0.0, 1.0, 20),
    ("two_cubes7", "barrier", 0.0, 0.8, 20),
    ("sphere_in_cube7", "barrier", 0.0, 0.8, 20),
    ("cube9", "shape_size", 0.0, 1.0, 10),
    ("two_cubes7", "untangle", 1e-3, 0.5, 10),
]


# Constrained boundary DOFs (2D closed-form entities), reference fp64 core:
# sweeps on grids whose boundary nodes slide on a Circle, an Ellipse, LineSegs
# and a LineRail, plus the entity Newton step and projection on random inputs
# -> ref_constrained.npz.
CASES_CON = {
    "disk_circle17": ("disk_on_curve", dict(n=17, seed=3)),
    "disk_ellipse17": ("disk_on_curve", dict(n=17, seed=4, ry=0.6)),
    "square_slide17": ("square_sliding", dict(n=17, seed=5)),
    "disk_circle33": ("disk_on_curve", dict(n=33, seed=6)),
    "disk_arcs17": ("disk_on_curve", dict(n=17, seed=7, arcs=True)),
    "cube_slide9": ("cube_sliding", dict(n=9, seed=8)),
    "disk_earcs17": ("disk_on_curve", dict(n=17, seed=9, ry=0.6, arcs=True)),
    "square_bezier17": ("square_bezier", dict(n=17, seed=10)),
    "cube_curved9": ("cube_curved", dict(n=9, seed=11)),
    "square_bspline17": ("square_bspline", dict(n=17, seed=12)),
    "square_composite17": ("square_composite", dict(n=17, seed=13)),
    "square_compbsp17": ("square_composite_bspline", dict(n=17, seed=14)),
}
RUNS_CON = [
    # (case, phase, delta, omega, n_sweeps)
    ("disk_circle17", "barrier", 0.0, 1.0, 30),
    ("disk_ellipse17", "barrier", 0.0, 0.8, 30),
    ("square_slide17", "barrier", 0.0, 1.0, 30),
    ("square_slide17", "shape_size", 0.0, 0.8, 20),
    ("disk_circle33", "barrier", 0.0, 1.0, 30),
    ("disk_circle17", "untangle", 1e-3, 0.5, 10),
    ("disk_arcs17", "barrier", 0.0, 1.0, 30),
    ("disk_arcs17", "barrier", 0.0, 0.8, 30),
    ("cube_slide9", "barrier", 0.0, 1.0, 20),
    ("cube_slide9", "barrier", 0.0, 0.8, 20),
    ("cube_slide9", "shape_size", 0.0, 1.0, 10),
    ("disk_earcs17", "barrier", 0.0, 1.0, 30),
    ("square_bezier17", "barrier", 0.0, 1.0, 30),
    ("square_bezier17", "barrier", 0.0, 0.8, 30),
    ("cube_curved9", "barrier", 0.0, 1.0, 20),
    ("cube_curved9", "barrier", 0.0, 0.8, 20),
    ("square_bspline17", "barrier", 0.0, 1.0, 30),
    ("square_bspline17", "barrier", 0.0, 0.8, 30),
    ("square_bspline17", "shape_size", 0.0, 1.0, 20),
    ("square_composite17", "barrier", 0.0, 1.0, 30),
    ("square_composite17", "barrier", 0.0, 0.8, 30),
    ("square_compbsp17", "barrier", 0.0, 1.0, 30),
    ("square_compbsp17", "barrier", 0.0, 0.8, 30),
    ("square_compbsp17", "shape_size", 0.0, 1.0, 20),
]
# FAS V-cycles on sliding-boundary grids: (case, phase, n_cycles, nu_pre, nu_post, nu_coarse, omega, max_levels)
FAS_RUNS_CON = [
    ("disk_circle33", "barrier", 4, 2, 2, 32, 0.8, 32),
    ("square_slide17", "barrier", 4, 2, 2, 32, 1.0, 32),
    ("disk_ellipse17", "barrier", 3, 2, 2, 32, 1.0, 3),
    ("disk_arcs17", "barrier", 3, 2, 2, 32, 1.0, 32),
    ("cube_slide9", "barrier", 3, 2, 2, 16, 1.0, 32),
    ("square_bezier17", "barrier", 3, 2, 2, 32, 1.0, 32),
    ("cube_curved9", "barrier", 3, 2, 2, 16, 1.0, 32),
    ("square_bspline17", "barrier", 3, 2, 2, 32, 1.0, 32),
    ("square_composite17", "barrier", 3, 2, 2, 32, 1.0, 32),
    ("square_compbsp17", "barrier", 3, 2, 2, 32, 1.0, 32),
]
# Soft terms (directional samples, 2D curvature windows) on seeded grids:
# name -> (configs builder, kwargs, with_soft_terms kwargs) -> ref_soft.npz.
CASES_SOFT = {
    "square_soft17": ("unit_square", dict(n=17, frac=0.25, seed=11), dict(seed=21)),
    "disk_oh_soft17": ("disk_oh", dict(n=17, frac=0.25, seed=12), dict(seed=22, block=1)),
    "slide_soft17": ("square_sliding", dict(n=17, seed=13), dict(seed=23)),
    "cube_soft7": ("unit_cube", dict(n=7, frac=0.15, seed=14), dict(seed=24, n_dir=30)),
    "square_soft33": ("unit_square", dict(n=33, frac=0.25, seed=15), dict(seed=25, n_dir=60, n_curv=40)),
}
RUNS_SOFT = [
    ("square_soft17", "barrier", 0.0, 1.0, 30),
    ("square_soft17", "barrier", 0.0, 0.8, 30),
    ("square_soft17", "shape_size", 0.0, 1.0, 20),
    ("square_soft17", "untangle", 1e-3, 0.5, 10),
    ("disk_oh_soft17", "barrier", 0.0, 1.0, 30),
    ("slide_soft17", "barrier", 0.0, 1.0, 30),
    ("cube_soft7", "barrier", 0.0, 1.0, 15),
    ("cube_soft7", "barrier", 0.0, 0.8, 15),
]
# control nets on soft-term grids: (case, block, ctrl shape, n_outer)
CONTROL_SOFT = [("square_soft17", 0, (6, 6), 8), ("disk_oh_soft17", 1, (6, 6), 8)]
FAS_RUNS_SOFT = [
    ("square_soft33", "barrier", 3, 2, 2, 32, 1.0, 32),
    ("disk_oh_soft17", "barrier", 3, 2, 2, 32, 0.8, 32),
]
ENTITY_RECORDS = {
    1: (0.1, -0.2, 0.9, 0.4),
    2: (0.2, -0.1, 0.7, 0.0),
    3: (-0.1, 0.3, 0.8, 0.45),
    15: (0.0, 0.0, 0.6, 0.3),
    6: (0.1, -0.05, 0.8, -2.6, 1.9, 0.0),
    7: (0.05, 0.1, 0.9, 0.5, 0.4, -1.0, 2.2, 0.0),
    8: (-0.2, 0.1, 0.4, 0.9, 1.0, -0.1, 0.1, 0.95),
    9: (-0.3, -0.2, 0.0, 0.8, 0.7, -0.6, 1.1, 0.3, 0.0, 1.0),
}


def case_grid(name: str):
    from egg_b200 import configs

    if name in CASES_SOFT:
        fn, kw, skw = CASES_SOFT[name]
        return configs.with_soft_terms(getattr(configs, fn)(**kw), **skw)
    if name in CASES_CON:
        fn, kw = CASES_CON[name]
        return getattr(configs, fn)(**kw)
    fn, kw, _ = CASES[name]
    return getattr(configs, fn)(**kw)


def _constrained_runs() -> dict:
    from oracle import oracle

    ref = oracle.load_ref("fp64")
    if ref is None:
        raise SystemExit("oracle/_ref/fp64 missing: run oracle/build_ref.sh first")
    out = {}
    for case, phase, delta, omega, n in RUNS_CON:
        g = case_grid(case)
        ctx, st = g.wire(), g.structured()
        X1, e1, m1 = ref.cpp_structured_sweep(ctx, st, g.X_flat(), 1, device="cpu", phase=phase,
                                               delta=delta, omega=omega, report_every=1, dim=g.d)
        Xn, en, mn = ref.cpp_structured_sweep(ctx, st, g.X_flat(), n, device="cpu", phase=phase,
                                               delta=delta, omega=omega, report_every=1, dim=g.d)
        key = f"{case}/{phase}/{omega}"
        out[key + "/X1"] = X1
        out[key + "/Xn"] = Xn
        out[key + "/E"] = en
        out[key + "/M"] = mn
    for case, phase, nc, npre, npost, ncoarse, omega, ml in FAS_RUNS_CON:
        g = case_grid(case)
        sess = ref.CppStructuredSweepSession(g.wire(), g.structured(), g.X_flat(), device="cpu", dim=g.d)
        E, M = sess.run_fas(nc, nu_pre=npre, nu_post=npost, nu_coarse=ncoarse, omega=omega, max_levels=ml,
                            phase=phase)
        key = f"fas/{case}/{phase}/{ml}"
        out[key + "/E"] = E
        out[key + "/M"] = M
        out[key + "/X"] = sess.get_X()
    rng3 = np.random.default_rng(37)
    # a session run in two calls: each call's first sweep projects cold
    g = case_grid("disk_arcs17")
    sess = ref.CppStructuredSweepSession(g.wire(), g.structured(), g.X_flat(), device="cpu", dim=2)
    e_a, _ = sess.run(10, report_every=1)
    e_b, _ = sess.run(20, report_every=1)
    out["twocalls/disk_arcs17/E"] = np.concatenate([e_a, e_b])
    out["twocalls/disk_arcs17/X"] = sess.get_X()
    # B-spline seeds: two run calls, then a fresh session from the positions
    # reached (positions uploaded anew: seeds cold) and a third call
    g = case_grid("square_bspline17")
    sess = ref.CppStructuredSweepSession(g.wire(), g.structured(), g.X_flat(), device="cpu", dim=2)
    e_a, _ = sess.run(7, report_every=1)
    e_b, _ = sess.run(12, report_every=1)
    sess = ref.CppStructuredSweepSession(g.wire(), g.structured(), sess.get_X(), device="cpu", dim=2)
    e_c, _ = sess.run(6, report_every=1)
    out["seeds/square_bspline17/E"] = np.concatenate([e_a, e_b, e_c])
    out["seeds/square_bspline17/X"] = sess.get_X()
    for case in ("cube_slide9", "cube_curved9"):
        g = case_grid(case)
        sess = ref.CppStructuredSweepSession(g.wire(), g.structured(), g.X_flat(), device="cpu", dim=3)
        e_a, _ = sess.run(5, report_every=1)
        e_b, _ = sess.run(10, report_every=1)
        out[f"twocalls/{case}/E"] = np.concatenate([e_a, e_b])
        out[f"twocalls/{case}/X"] = sess.get_X()
    # 3D projections: the reference's own batched projection
    c, sn = np.cos(0.4), np.sin(0.4)
    for tag, rec in ((5, (0.1, -0.2, 0.3, c, sn, 0.0, 0.0, 0.0, 1.0)), (16, (0.1, 0.0, -0.1, 0.7, 0.3, 0.2)),
                     (4, (0.2, 0.1, -0.3, 0.9, c, sn, 0.0, -sn, c, 0.0)),
                     (12, (0.1, 0.2, 0.0, c, 0.0, sn, 0.0, 1.0, 0.0, 0.7)),
                     (13, (0.1, 0.0, -0.1, 0.7, 0.3, 0.2, 0.1, 0.8))):
        Q = rng3.uniform(-0.5, 1.2, size=(64, 3))
        feet, _basis = ref.geometry_project_batch(Q, tag, np.array(rec), [])
        out[f"entity3/{tag}/params"] = np.array(rec)
        out[f"entity3/{tag}/pos"] = Q
        out[f"entity3/{tag}/foot"] = np.asarray(feet)
    rng = np.random.default_rng(31)
    for tag, rec in ENTITY_RECORDS.items():
        from egg_b200.wire import ENTITY_KINDS

        kf = ENTITY_KINDS[tag][1]
        params = np.array(rec[:kf])
        G = rng.normal(size=(64, 2))
        G[:4] *= 1e-17  # below the zero-gradient guard
        H = rng.normal(size=(64, 2, 2))
        H = H @ H.transpose(0, 2, 1) + 0.1 * np.eye(2)
        H[4:8] = 0.0  # singular reduced system: the fallback step
        P = rng.uniform(-1.2, 1.4, size=(64, 2))
        steps = np.array([ref.newton_step(G[i], H[i].ravel(), P[i], tag, params) for i in range(64)])
        feet = np.array([ref.geometry_project(P[i], tag, params) for i in range(64)])
        out[f"entity/{tag}/params"] = params
        out[f"entity/{tag}/grad"] = G
        out[f"entity/{tag}/hess"] = H.reshape(64, 4)
        out[f"entity/{tag}/pos"] = P
        out[f"entity/{tag}/step"] = steps
        out[f"entity/{tag}/foot"] = feet
    return out


def _soft_runs(ref_root: Path) -> dict:
    """Reference-core sweeps and FAS cycles on the soft-term grids, plus the
    reference's own per-DOF and whole-sample tables for the wire check."""
    sys.path.insert(0, str(ref_root))
    from egg.smoothing.directional import DirectionalSamples, directional_dof_table, directional_energy_table
    from egg.smoothing.interface_c2 import CurvatureWindows, curvature_dof_table

    from oracle import oracle

    ref = oracle.load_ref("fp64")
    if ref is None:
        raise SystemExit("oracle/_ref/fp64 missing: run oracle/build_ref.sh first")
    out = {}
    for case in CASES_SOFT:
        g = case_grid(case)
        moving = g.free.copy()
        moving[list(g.constraints)] = True
        ds = g.soft["directional"]
        smp = DirectionalSamples(nodes=ds["nodes"], kind=ds["kind"], ref=ds["ref"], axis=ds["axis"],
                                 weight=ds["weight"], eps=ds["eps"])
        tabs = {"dof": directional_dof_table(moving, smp), "es": directional_energy_table(smp)}
        if "curvature" in g.soft:
            cw = g.soft["curvature"]
            tabs["dof_curv"] = curvature_dof_table(moving, CurvatureWindows(nodes=cw["nodes"], weight=cw["weight"]))
        for part, t in tabs.items():
            for k, v in t.items():
                out[f"table/{case}/{part}/{k}"] = np.asarray(v)
    for case, phase, delta, omega, n in RUNS_SOFT:
        g = case_grid(case)
        ctx, st = g.wire(), g.structured()
        X1, _e1, _m1 = ref.cpp_structured_sweep(ctx, st, g.X_flat(), 1, device="cpu", phase=phase,
                                                 delta=delta, omega=omega, report_every=1, dim=g.d)
        Xn, en, mn = ref.cpp_structured_sweep(ctx, st, g.X_flat(), n, device="cpu", phase=phase,
                                               delta=delta, omega=omega, report_every=1, dim=g.d)
        key = f"{case}/{phase}/{omega}"
        out[key + "/X1"] = X1
        out[key + "/Xn"] = Xn
        out[key + "/E"] = en
        out[key + "/M"] = mn
    from egg.geometry.control_net import tensor_map
    from egg.smoothing.control_backend import build_control_wire
    from egg.smoothing.control_ref import boolean_sum_b, boundary_ctrl_mask, fit_control_net

    for case, blk, ctrl, n_outer in CONTROL_SOFT:
        g = case_grid(case)
        ids = g.blocks[blk]
        X0b = g.X[ids.reshape(-1)].reshape(ids.shape + (g.d,))
        cmap = tensor_map(ids.shape, ctrl, degree=3)
        C0 = fit_control_net(cmap, X0b)
        wire = build_control_wire(cmap, C0, ~boundary_ctrl_mask(tuple(ctrl)), boolean_sum_b(cmap, C0, X0b),
                                  block=blk)
        for k, v in wire.items():
            out[f"control/{case}/wire/{k}"] = np.asarray(v)
        sess = ref.CppStructuredSweepSession(g.wire(), g.structured(), g.X_flat(), device="cpu", dim=g.d,
                                             control=wire)
        rep = sess.run_control(n_outer)
        for k in ("energies", "mindets", "alphas", "pcg_iters"):
            out[f"control/{case}/{k}"] = np.asarray(rep[k], dtype=float)
        out[f"control/{case}/iters"] = np.int64(rep["iters"])
        out[f"control/{case}/X"] = np.asarray(sess.get_X())
        out[f"control/{case}/C"] = np.asarray(sess.get_C())
        print(case, "control iters", rep["iters"], "E", rep["energies"][0], "->", rep["energies"][-1])
    for case, phase, nc, npre, npost, ncoarse, omega, ml in FAS_RUNS_SOFT:
        g = case_grid(case)
        sess = ref.CppStructuredSweepSession(g.wire(), g.structured(), g.X_flat(), device="cpu", dim=g.d)
        E, M = sess.run_fas(nc, nu_pre=npre, nu_post=npost, nu_coarse=ncoarse, omega=omega, max_levels=ml,
                            phase=phase)
        key = f"fas/{case}/{phase}/{ml}"
        out[key + "/E"] = E
        out[key + "/M"] = M
        out[key + "/X"] = sess.get_X()
    return out


def gen_reference_soft(ref_root: Path) -> None:
    out = _soft_runs(ref_root)
    np.savez_compressed(HERE / "ref_soft.npz", **out)
    print(f"ref_soft.npz: {len(out)} arrays")


def gen_reference_constrained() -> None:
    out = _constrained_runs()
    np.savez_compressed(HERE / "ref_constrained.npz", **out)
    print(f"ref_constrained.npz: {len(out)} arrays")


def _runs_for(prec: str) -> dict:
    from oracle import oracle

    ref = oracle.load_ref(prec)
    if ref is None:
        raise SystemExit(f"oracle/_ref/{prec} missing: run oracle/build_ref.sh first")
    assert bool(ref.REAL_IS_FLOAT) == (prec == "fp32")
    out = {}
    for case, phase, delta, omega, n in RUNS + RUNS3:
        g = case_grid(case)
        ctx, st = g.wire(), g.structured()
        X1, e1, m1 = ref.cpp_structured_sweep(ctx, st, g.X_flat(), 1, device="cpu", phase=phase,
                                               delta=delta, omega=omega, report_every=1, dim=g.d)
        Xn, en, mn = ref.cpp_structured_sweep(ctx, st, g.X_flat(), n, device="cpu", phase=phase,
                                               delta=delta, omega=omega, report_every=1, dim=g.d)
        key = f"{prec}/{case}/{phase}/{omega}"
        out[key + "/X1"] = X1
        out[key + "/Xn"] = Xn
        out[key + "/E"] = en
        out[key + "/M"] = mn
        out[key + "/E1"] = e1
    for case, phase, nc, npre, npost, ncoarse, omega, ml in FAS_RUNS:
        g = case_grid(case)
        sess = ref.CppStructuredSweepSession(g.wire(), g.structured(), g.X_flat(), device="cpu", dim=g.d)
        E, M = sess.run_fas(nc, nu_pre=npre, nu_post=npost, nu_coarse=ncoarse, omega=omega, max_levels=ml,
                            phase=phase)
        key = f"{prec}/fas/{case}/{phase}/{ml}"
        out[key + "/E"] = E
        out[key + "/M"] = M
        out[key + "/X"] = sess.get_X()
        levels = sess.mg_levels()
        out[key + "/levels"] = np.array([[list(t) for t in lv] for lv in levels], dtype=np.int32).reshape(
            len(levels), -1)
    return out


def gen_reference_runs() -> None:
    """One process per precision: two extension modules named cpp_core cannot
    coexist in one interpreter."""
    import subprocess
    import tempfile

    out = {}
    for prec in ("fp64", "fp32"):
        with tempfile.TemporaryDirectory() as td:
            f = Path(td) / "runs.npz"
            subprocess.run([sys.executable, __file__, "--runs", prec, str(f)], check=True)
            out.update(dict(np.load(f)))
    np.savez_compressed(HERE / "ref_sweeps.npz", **out)
    print(f"ref_sweeps.npz: {len(out)} arrays")


def gen_reference_wire(ref_root: Path) -> None:
    """The reference's own wire builders on a small multi-block grid."""
    sys.path.insert(0, str(ref_root))
    from egg.smoothing.cpp_backend import build_structured_context_from_block_maps, structured_arrays
    from egg.smoothing.flat_context import build_flat_context

    g = case_grid("disk_oh17")
    out = {}
    for tag, w in (("eye", np.eye(2)), ("aniso", np.array([[1.0, 0.2], [0.0, 1.3]]))):
        ctx = build_flat_context([np.asarray(b) for b in g.blocks], g.free, {}, 2, w_inv=w)
        for k, v in ctx["groups"][0].items():
            if isinstance(v, np.ndarray):
                out[f"{tag}/group/{k}"] = v
        for k, v in ctx["energy_stencil"].items():
            if isinstance(v, np.ndarray):
                out[f"{tag}/es/{k}"] = v
    st = structured_arrays(build_structured_context_from_block_maps(2, g.blocks))
    for k, v in st.items():
        if isinstance(v, list):
            for i, a in enumerate(v):
                out[f"st/{k}/{i}"] = np.asarray(a)
        else:
            out[f"st/{k}"] = np.asarray(v)
    np.savez_compressed(HERE / "ref_wire_disk_oh17.npz", **out)
    print(f"ref_wire_disk_oh17.npz: {len(out)} arrays")


# Control-net runs: (grid source, ctrl shape, controlled block, phase, n_outer,
# run_control options, also run the reference's NumPy dense-GN oracle).
CONTROL_CASES = {
    "wavy13": ("wavy", dict(n=13), (6, 6), 0, "barrier", 30,
               dict(pcg_max_iter=500, pcg_rtol=1e-12, pcg_forcing=False), True),
    "wavy9": ("wavy", dict(n=9), (5, 5), 0, "barrier", 5, {}, False),
    "wavy13ss": ("wavy", dict(n=13), (6, 6), 0, "shape_size", 12, {}, False),
    "cube9c": ("unit_cube", dict(n=9, frac=0.15, seed=31), (5, 5, 5), 0, "barrier", 8, {}, False),
    "disk17c": ("disk_oh", dict(n=17, frac=0.25, seed=2), (6, 6), 0, "barrier", 8, {}, False),
    # sessions with constrained boundary DOFs (sliding sides; a circle outside the net's block)
    "slide17c": ("square_sliding", dict(n=17, seed=5), (6, 6), 0, "barrier", 8, {}, False),
    "circle17c": ("disk_on_curve", dict(n=17, seed=3), (6, 6), 0, "barrier", 8, {}, False),
}


def control_case_grid(name: str, fx) -> "object":
    """The case's grid as an egg_b200 configs.Grid (wavy grids come from the
    fixture, which stores the reference-built nodes)."""
    from egg_b200 import configs

    src, kw, *_ = CONTROL_CASES[name]
    if src != "wavy":
        return getattr(configs, src)(**kw)
    ids = np.asarray(fx[f"{name}/ids"])
    X = np.asarray(fx[f"{name}/X0"])
    free = np.zeros(X.shape[0], dtype=bool)
    free[ids[1:-1, 1:-1].reshape(-1)] = True
    return configs.Grid(name, 2, [ids], X, free, {})


def _control_runs(ref_root: Path) -> dict:
    sys.path.insert(0, str(ref_root))
    from egg.geometry.control_net import tensor_map
    from egg.smoothing.control_backend import build_control_wire
    from egg.smoothing.control_ref import (boolean_sum_b, boundary_ctrl_mask, build_control_ref,
                                           fit_control_net, run_control_ref)
    from egg.smoothing.targets import IdentityTarget
    from tests.smoothing.test_control_ref import _make_wavy_grid

    from oracle import oracle

    ref = oracle.load_ref("fp64")
    out = {}
    for name, (src, kw, ctrl, blk, phase, n_outer, opts, numpy_ref) in CONTROL_CASES.items():
        if src == "wavy":
            rg = _make_wavy_grid(**kw)
            out[f"{name}/X0"] = np.asarray(rg.global_nodes, dtype=float)
            out[f"{name}/ids"] = np.asarray(rg.block_dof_maps[0], dtype=np.int64)
        g = control_case_grid(name, out)
        ids = g.blocks[blk]
        X0b = g.X[ids.reshape(-1)].reshape(ids.shape + (g.d,))
        cmap = tensor_map(ids.shape, ctrl, degree=3)
        C0 = fit_control_net(cmap, X0b)
        bf = boolean_sum_b(cmap, C0, X0b)
        wire = build_control_wire(cmap, C0, ~boundary_ctrl_mask(tuple(ctrl)), bf, block=blk)
        for k, v in wire.items():
            out[f"{name}/wire/{k}"] = np.asarray(v)
        s = ref.CppStructuredSweepSession(g.wire(), g.structured(), g.X_flat(), device="cpu", dim=g.d,
                                          control=wire)
        rep = s.run_control(n_outer, phase=phase, **opts)
        for k in ("energies", "mindets", "alphas", "pcg_iters", "pcg_relres"):
            out[f"{name}/ref/{k}"] = np.asarray(rep[k], dtype=float)
        out[f"{name}/ref/iters"] = np.int64(rep["iters"])
        out[f"{name}/ref/converged"] = np.int64(bool(rep["converged"]))
        out[f"{name}/ref/X"] = np.asarray(s.get_X())
        out[f"{name}/ref/C"] = np.asarray(s.get_C())
        print(name, "iters", rep["iters"], "E", rep["energies"][0], "->", rep["energies"][-1])
        if numpy_ref:
            rg2 = _make_wavy_grid(**kw)
            cref = build_control_ref(rg2, IdentityTarget(d=2), ctrl)
            r2 = run_control_ref(cref, max_outer=n_outer)
            out[f"{name}/numpy/energies"] = np.asarray(r2["energies"], dtype=float)
            out[f"{name}/numpy/iters"] = np.int64(r2["iters"])
            out[f"{name}/numpy/X"] = np.asarray(rg2.global_nodes, dtype=float).reshape(-1)
            print(name, "numpy iters", r2["iters"], "E", r2["energies"][-1])
    return out


def gen_reference_control(ref_root: Path) -> None:
    import subprocess
    import tempfile

    with tempfile.TemporaryDirectory() as td:
        f = Path(td) / "control.npz"
        subprocess.run([sys.executable, __file__, "--control", str(ref_root), str(f)], check=True)
        out = dict(np.load(f))
    np.savez_compressed(HERE / "ref_control.npz", **out)
    print(f"ref_control.npz: {len(out)} arrays")


# ---------------------------------------------------------------------------
# The benchmark configurations at their own sizes, run by the reference core
# (fp64 build): C1 exactly, C3 at 1025^2 (untangle schedule, then shape+size),
# C4 as the 7-block sphere-in-cube at 33^3 (untangle, FAS V(2,2), 4 levels),
# C5 as 32 batched multi-block meshes.  Positions of the larger cases are kept
# at every CONFIG_STRIDE-th node to keep the fixture small.
# ---------------------------------------------------------------------------
CONFIG_STRIDE = {"c3": 101, "c4": 47, "c5": 151}
C3_SHAPE_SIZE_SWEEPS = 100
C4_CYCLES = 4
C5_MESHES = 32


def _ref_untangle(make_session, X, mindet0, *, sweeps_per_delta=20, delta0_factor=2.0, shrink=0.8, max_outer=60,
                  margin=1e-9, omega=0.5):
    """The delta-continuation schedule of egg/smoothing/cpp_backend.py:773-848
    on a reference-core session; returns (session, per-step min det, deltas)."""
    mds, deltas = [], []
    if mindet0 > margin:
        return None, mds, deltas
    sess = make_session(X)
    delta = delta0_factor * max(abs(mindet0), 1e-12)
    for _ in range(max_outer):
        _e, m = sess.run(sweeps_per_delta, phase="untangle", delta=delta, omega=omega)
        mds.append(float(np.asarray(m)[-1]))
        deltas.append(delta)
        if mds[-1] > margin:
            break
        delta *= shrink
    return sess, mds, deltas


def _config_runs() -> dict:
    import time

    from egg_b200 import configs
    from oracle import oracle

    ref = oracle.load_ref("fp64")
    if ref is None:
        raise SystemExit("oracle/_ref/fp64 missing: run oracle/build_ref.sh first")
    out = {}
    t0 = time.perf_counter()
    # C1: disk O-H 5 x 65^2, +-0.25h, shape, 40 sweeps
    g = configs.disk_oh(65, frac=0.25, seed=0)
    ctx, st = g.wire(), g.structured()
    X1, e1, _ = ref.cpp_structured_sweep(ctx, st, g.X_flat(), 1, device="cpu", phase="barrier", report_every=1, dim=2)
    Xn, E, M = ref.cpp_structured_sweep(ctx, st, g.X_flat(), 40, device="cpu", phase="barrier", report_every=1,
                                        dim=2)
    out.update({"c1/X1": X1, "c1/E1": e1, "c1/X40": Xn, "c1/E": E, "c1/M": M})
    print(f"C1 {time.perf_counter() - t0:.1f}s", flush=True)
    # C3: 1025^2, ~5% inverted: untangle schedule, then shape+size (mean-size target)
    g = configs.tangled_square(1025, target=0.05, seed=0)
    md0 = float(configs.grid_mindet(g.blocks, g.X).min())
    sa, mds, deltas = _ref_untangle(
        lambda X: ref.CppStructuredSweepSession(g.wire(), g.structured(), X, device="cpu"), g.X_flat(),
        md0)
    Xu = sa.get_X()
    sb = ref.CppStructuredSweepSession(g.wire(w_inv=configs.mean_size_w_inv(g.blocks, g.X)),
                                       g.structured(), Xu, device="cpu")
    E, M = sb.run(C3_SHAPE_SIZE_SWEEPS, phase="shape_size", report_every=10)
    k = CONFIG_STRIDE["c3"]
    out.update({"c3/mindet0": np.array(md0), "c3/untangle_mindets": np.array(mds), "c3/deltas": np.array(deltas),
                "c3/Xu": Xu.reshape(-1, 2)[::k].copy(), "c3/E": E, "c3/M": M,
                "c3/X": sb.get_X().reshape(-1, 2)[::k].copy()})
    print(f"C3 {time.perf_counter() - t0:.1f}s, {len(mds)} delta steps", flush=True)
    # C4: 7-block sphere-in-cube 33^3, +-0.2h: untangle, then FAS V(2,2), 4 levels
    g = configs.sphere_in_cube(33, frac=0.2, seed=0)
    md0 = float(configs.grid_mindet(g.blocks, g.X, 3).min())

    def make(X):
        return ref.CppStructuredSweepSession(g.wire(), g.structured(), X, device="cpu", dim=3)

    sa, mds, deltas = _ref_untangle(make, g.X_flat(), md0)
    Xu = sa.get_X() if sa is not None else g.X_flat()
    sf = make(Xu)
    E, M = sf.run_fas(C4_CYCLES, nu_pre=2, nu_post=2, max_levels=4)
    k = CONFIG_STRIDE["c4"]
    lv = sf.mg_levels()
    out.update({"c4/mindet0": np.array(md0), "c4/untangle_mindets": np.array(mds), "c4/deltas": np.array(deltas),
                "c4/E": E, "c4/M": M, "c4/X": sf.get_X().reshape(-1, 3)[::k].copy(),
                "c4/levels": np.array([[list(t) for t in x] for x in lv], dtype=np.int32).reshape(len(lv), -1)})
    print(f"C4 {time.perf_counter() - t0:.1f}s, {len(mds)} delta steps", flush=True)
    # C5: 32 multi-block meshes, 20 sweeps, each by its own reference session
    Es, Ms, Xs = [], [], []
    for gm in configs.batch_meshes(C5_MESHES, seed=0):
        Xo, E, M = ref.cpp_structured_sweep(gm.wire(), gm.structured(), gm.X_flat(), 20, device="cpu",
                                            phase="barrier", report_every=10, dim=2)
        Es.append(E)
        Ms.append(M)
        Xs.append(Xo.reshape(-1, 2))
    k = CONFIG_STRIDE["c5"]
    out.update({"c5/E": np.array(Es), "c5/M": np.array(Ms), "c5/X": np.concatenate(Xs)[::k].copy()})
    print(f"C5 {time.perf_counter() - t0:.1f}s", flush=True)
    return out


def gen_reference_configs() -> None:
    out = _config_runs()
    np.savez_compressed(HERE / "ref_configs.npz", **out)
    print(f"ref_configs.npz: {len(out)} arrays")


if __name__ == "__main__" and len(sys.argv) == 2 and sys.argv[1] == "--configs":
    gen_reference_configs()
    raise SystemExit(0)

# ---------------------------------------------------------------------------
# The reference core's remaining free functions (src/bindings.cpp:1819-2100):
# geometry_tangent on the closed-form curves, geometry_project_batch on one
# entity row of every constrained test grid, energy_mindet on the golden
# patches, directional_eval on seeded sample tables (2D and 3D).
# ---------------------------------------------------------------------------
FREE_BATCH_CASES = ["disk_arcs17", "disk_earcs17", "square_slide17", "square_bezier17", "square_bspline17",
                    "square_composite17", "square_compbsp17", "cube_slide9", "cube_curved9", "disk_circle17",
                    "disk_ellipse17"]


def _entity_rows(g):
    """(tag, record row, per-row seg list) of the first DOF of every entity
    partition of a grid's wire, in the reference's single-row encoding."""
    out = []
    for name, ed in g.wire()["groups"][0]["entities"].items():
        tag = int(ed["tag"])
        if tag == 0:
            continue
        kf = int(ed["kFields"])
        rec = np.asarray(ed["records"], dtype=np.float64).reshape(-1, kf)[0]
        seg = []
        for sd in ed.get("seg", []):
            off = np.asarray(sd["off"])
            seg.append({"data": np.asarray(sd["data"], dtype=np.float64)[off[0]:off[1]].copy(),
                        "off": np.array([0, off[1] - off[0]], dtype=np.int32)})
        out.append((name, tag, rec, seg))
    return out


def _free_runs() -> dict:
    from egg_b200.wire import ENTITY_KINDS
    from oracle import oracle

    ref = oracle.load_ref("fp64")
    if ref is None:
        raise SystemExit("oracle/_ref/fp64 missing: run oracle/build_ref.sh first")
    rng = np.random.default_rng(21)
    out = {}
    for tag, rec in ENTITY_RECORDS.items():
        params = np.array(rec[: ENTITY_KINDS[tag][1]])
        P = rng.uniform(-1.2, 1.4, size=(48, 2))
        out[f"tangent/{tag}/params"] = params
        out[f"tangent/{tag}/pos"] = P
        out[f"tangent/{tag}/t"] = np.array([ref.geometry_tangent(P[i], tag, params) for i in range(len(P))])
    k = 0
    for case in FREE_BATCH_CASES:
        g = case_grid(case)
        lo, hi = g.X.min(axis=0), g.X.max(axis=0)
        for name, tag, rec, seg in _entity_rows(g):
            q = lo + (hi - lo) * rng.uniform(-0.1, 1.1, size=(40, g.d))
            feet, basis = ref.geometry_project_batch(q, tag, rec, seg)
            key = f"batch/{k}/"
            out[key + "case"] = np.array(case)
            out[key + "tag"] = np.array(tag)
            out[key + "rec"] = rec
            for j, sd in enumerate(seg):
                out[key + f"seg{j}_data"] = sd["data"]
                out[key + f"seg{j}_off"] = sd["off"]
            out[key + "nseg"] = np.array(len(seg))
            out[key + "q"] = q
            out[key + "feet"] = np.asarray(feet)
            out[key + "basis"] = np.asarray(basis)
            k += 1
    out["batch/count"] = np.array(k)
    patches = json.loads((HERE / "golden_patch.json").read_text())["records"]
    em = []
    for r in patches:
        P, n = int(r["P"]), int(r["n_nodes"])
        em.append(ref.energy_mindet(np.array(r["X"][: 2 * n]), np.array(r["gc"][:P], dtype=np.int32),
                                    np.array(r["gn0"][:P], dtype=np.int32), np.array(r["gn1"][:P], dtype=np.int32),
                                    np.array(r["s0"][:P]), np.array(r["s1"][:P]), np.array(r["W_inv"][: 4 * P])))
    out["energy_mindet"] = np.array(em)
    for d in (2, 3):
        nn, ns = 40, 60
        X = rng.normal(size=(nn, d))
        kind = rng.integers(0, 3, size=ns).astype(np.int32)
        nodes = np.full((ns, 4), -1, dtype=np.int32)
        for i in range(ns):
            ar = 3 if kind[i] == 1 else 2
            nodes[i, :ar] = rng.choice(nn, size=ar, replace=False)
        refv = rng.normal(size=(ns, d))
        refv /= np.linalg.norm(refv, axis=1, keepdims=True)
        w = rng.uniform(0.1, 2.0, size=ns)
        e, gr = ref.directional_eval(X, nodes, kind, refv, w, 1e-3)
        key = f"dir{d}/"
        out.update({key + "X": X, key + "nodes": nodes, key + "kind": kind, key + "ref": refv, key + "w": w,
                    key + "e": np.array(e), key + "g": np.asarray(gr)})
    return out


def gen_reference_free() -> None:
    out = _free_runs()
    np.savez_compressed(HERE / "ref_free.npz", **out)
    print(f"ref_free.npz: {len(out)} arrays")


# B-spline / NURBS surfaces (entity tag 14), reference fp64 core: sweeps,
# two run calls (the seeds persist, each call's first sweep projects from
# them in world space), FAS, and the reference's batched projection onto a
# polynomial, a rational and a UV-trimmed surface -> ref_bsurf.npz.
BSURF_CASE = ("cube_bsurf", dict(n=9, seed=15))
BSURF_RUNS = [("barrier", 0.0, 1.0, 20), ("barrier", 0.0, 0.8, 20), ("shape_size", 0.0, 1.0, 10)]
# a trim polygon in the top surface's (u, v): an outer loop and a hole
BSURF_TRIM = [np.array([[0.05, 0.05], [0.95, 0.08], [0.9, 0.95], [0.1, 0.9]]),
              np.array([[0.4, 0.4], [0.6, 0.4], [0.55, 0.6]])]


def bsurf_entities():
    """(name, tag, record, seg) of the three projection surfaces."""
    from egg_b200 import configs

    top, side, w = configs.bsurf_nets()
    out = []
    for name, kw, net, wt, trim in (("poly", configs.BSURF_TOP, top, None, None),
                                    ("nurbs", configs.BSURF_SIDE, side, w, None),
                                    ("trimmed", configs.BSURF_TOP, top, None, BSURF_TRIM)):
        tag, rec, seg = configs._bsurf_entity(kw["pu"], kw["pv"], kw["ku"], kw["kv"], net, wt, trim)
        out.append((name, tag, np.asarray(rec), [{"data": np.asarray(a, dtype=np.float64),
                                                   "off": np.array([0, np.asarray(a).size], dtype=np.int32)}
                                                  for a in seg]))
    return out


def _bsurf_runs() -> dict:
    from egg_b200 import configs
    from oracle import oracle

    ref = oracle.load_ref("fp64")
    if ref is None:
        raise SystemExit("oracle/_ref/fp64 missing: run oracle/build_ref.sh first")
    out = {}
    g = getattr(configs, BSURF_CASE[0])(**BSURF_CASE[1])
    ctx, st = g.wire(), g.structured()
    for phase, delta, omega, n in BSURF_RUNS:
        X1, _e1, _m1 = ref.cpp_structured_sweep(ctx, st, g.X_flat(), 1, device="cpu", phase=phase, delta=delta,
                                                omega=omega, report_every=1, dim=3)
        Xn, en, mn = ref.cpp_structured_sweep(ctx, st, g.X_flat(), n, device="cpu", phase=phase, delta=delta,
                                              omega=omega, report_every=1, dim=3)
        key = f"{phase}/{omega}"
        out[key + "/X1"] = X1
        out[key + "/Xn"] = Xn
        out[key + "/E"] = en
        out[key + "/M"] = mn
    sess = ref.CppStructuredSweepSession(ctx, st, g.X_flat(), device="cpu", dim=3)
    e_a, _ = sess.run(5, report_every=1)
    e_b, _ = sess.run(10, report_every=1)
    out["twocalls/E"] = np.concatenate([e_a, e_b])
    out["twocalls/X"] = sess.get_X()
    sess = ref.CppStructuredSweepSession(ctx, st, g.X_flat(), device="cpu", dim=3)
    E, M = sess.run_fas(3, nu_pre=2, nu_post=2, nu_coarse=16, omega=1.0, max_levels=32, phase="barrier")
    out["fas/E"] = E
    out["fas/M"] = M
    out["fas/X"] = sess.get_X()
    rng = np.random.default_rng(41)
    for name, tag, rec, seg in bsurf_entities():
        Q = rng.uniform(-0.2, 1.2, size=(48, 3))
        Q[:, 2 if name != "nurbs" else 0] = 1.0 + rng.uniform(-0.3, 0.3, 48)
        feet, basis = ref.geometry_project_batch(Q, tag, rec, seg)
        out[f"project/{name}/q"] = Q
        out[f"project/{name}/foot"] = np.asarray(feet)
        out[f"project/{name}/basis"] = np.asarray(basis)
    return out


def gen_reference_bsurf() -> None:
    out = _bsurf_runs()
    np.savez_compressed(HERE / "ref_bsurf.npz", **out)
    print(f"ref_bsurf.npz: {len(out)} arrays")


if __name__ == "__main__" and len(sys.argv) == 2 and sys.argv[1] == "--bsurf":
    gen_reference_bsurf()
    raise SystemExit(0)

if __name__ == "__main__" and len(sys.argv) == 2 and sys.argv[1] == "--free":
    gen_reference_free()
    raise SystemExit(0)

if __name__ == "__main__" and len(sys.argv) == 4 and sys.argv[1] == "--control":
    np.savez(sys.argv[3], **_control_runs(Path(sys.argv[2])))
    raise SystemExit(0)

if __name__ == "__main__" and len(sys.argv) == 4 and sys.argv[1] == "--runs":
    np.savez(sys.argv[3], **_runs_for(sys.argv[2]))
    raise SystemExit(0)

if __name__ == "__main__" and len(sys.argv) in (2, 3) and sys.argv[1] == "--soft":
    gen_reference_soft(Path(sys.argv[2]) if len(sys.argv) == 3 else _ref_root())
    raise SystemExit(0)

if __name__ == "__main__" and len(sys.argv) == 2 and sys.argv[1] == "--constrained":
    gen_reference_constrained()
    raise SystemExit(0)

if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    ref_root = Path(args[0]) if args else _ref_root()
    gen_reference_vectors(ref_root)
    gen_reference_runs()
    gen_reference_wire(ref_root)
    gen_reference_control(ref_root)
    gen_reference_constrained()
    gen_reference_soft(ref_root)
    gen_reference_configs()
    gen_reference_free()
    gen_reference_bsurf()
