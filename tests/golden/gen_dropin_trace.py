"""Record the reference's own Python drivers talking to a cpp_core module.

The reference's smoothing drivers (``egg/smoothing/cpp_backend.py``:
``CppStructuredSweepSession``, ``cpp_structured_sweep``, ``cpp_untangle``;
``egg/pipeline.py:510-527`` ``_cpp_reduce``) reach the compiled core only
through ``egg._cpp.cpp_core``.  This script runs them, unmodified, from the
reference checkout with ``egg._cpp.cpp_core`` replaced by a recording proxy
around the reference core built from source with its parallel loops run
serially in the race-free order (``oracle/_ref/fp64snap``).  The plain OpenMP
build is not a usable recorder here: on these multi-block grids the
reference's fused ghost-fill + shared-node-refresh launch
(``src/structured_halo.hpp:215-236``) reads non-owner copies while they are
refreshed, and its positions after two sweeps on the O-grid differ by 2.2e-5
between 8 threads and 1 or 2 threads.  Every
call that crosses the module boundary -- its arguments exactly as the driver
built them, and the reference core's results -- goes to
``tests/golden/ref_dropin.pkl.gz``.

``tests/test_dropin_gpu.py`` replays that trace against ``egg_b200.cpp_core``
on the GPU: the drop-in boundary is then exercised by the very calls the
reference's drivers make, which the GPU host cannot generate itself (the
reference's Python does not travel there).

    python tests/golden/gen_dropin_trace.py [REFERENCE_ROOT]          # ref_dropin.pkl.gz
    python tests/golden/gen_dropin_trace.py --topo [REFERENCE_ROOT]   # ref_dropin_topo.pkl.gz
    python tests/golden/gen_dropin_trace.py --walls [REFERENCE_ROOT]  # ref_dropin_walls.pkl.gz
    python tests/golden/gen_dropin_trace.py --slides [REFERENCE_ROOT] # ref_dropin_slides.pkl.gz

(default: ``$EGG_REFERENCE_ROOT`` or a ``reference`` checkout beside this
repository).  Test infrastructure only.
"""

from __future__ import annotations

import gzip
import pickle
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

TRACE = HERE / "ref_dropin.pkl.gz"


def _copy(v):
    """Deep copy of an argument or result (numpy arrays, dicts, lists, tuples)."""
    if isinstance(v, np.ndarray):
        return v.copy()
    if isinstance(v, dict):
        return {k: _copy(x) for k, x in v.items()}
    if isinstance(v, list):
        return [_copy(x) for x in v]
    if isinstance(v, tuple):
        return tuple(_copy(x) for x in v)
    if isinstance(v, (np.floating, np.integer)):
        return v.item()
    return v


class Recorder:
    """Builds the proxy module and collects the trace.  A session that the
    driver opens on the reference's host device (``device="cpu"``) is
    recorded with ``device="auto"``: the replay runs it on the GPU."""

    def __init__(self, ref):
        self.ref = ref
        self.events: list[dict] = []
        self.scenario = ""
        self._next_sid = 0

    def log(self, **ev):
        ev["scenario"] = self.scenario
        self.events.append(ev)

    def module(self) -> types.ModuleType:
        rec = self
        ref = self.ref
        mod = types.ModuleType("egg._cpp.cpp_core")
        for name in dir(ref):
            if name.startswith("_") or name == "CppStructuredSweepSession":
                continue
            obj = getattr(ref, name)
            if callable(obj):

                def fn(*args, _name=name, _obj=obj, **kwargs):
                    out = _obj(*args, **kwargs)
                    rec.log(op="fn", name=_name, args=_copy(args), kwargs=_copy(kwargs), result=_copy(out))
                    return out

                setattr(mod, name, fn)
            else:
                setattr(mod, name, obj)

        class CppStructuredSweepSession:
            def __init__(self, *args, **kwargs):
                self._s = ref.CppStructuredSweepSession(*args, **kwargs)
                self._sid = rec._next_sid
                rec._next_sid += 1
                kw = _copy(kwargs)
                if kw.get("device") == "cpu":
                    kw["device"] = "auto"
                rec.log(op="new", sid=self._sid, args=_copy(args), kwargs=kw)

            def __getattr__(self, name):
                attr = getattr(self._s, name)
                if not callable(attr):
                    return attr

                def method(*args, **kwargs):
                    out = attr(*args, **kwargs)
                    rec.log(op="call", sid=self._sid, name=name, args=_copy(args), kwargs=_copy(kwargs),
                            result=_copy(out))
                    return out

                return method

        mod.CppStructuredSweepSession = CppStructuredSweepSession
        return mod


def _perturb(grid, seed: int, scale: float) -> np.ndarray:
    """Seeded normal noise on the free nodes that carry no boundary
    constraint, written back into the grid's global and per-block views."""
    rng = np.random.default_rng(seed)
    X = np.array(grid.global_nodes, dtype=np.float64)
    free = np.asarray(grid.free_mask, dtype=bool)
    movable = [i for i in range(X.shape[0]) if free[i] and i not in grid.dof_constraints]
    X[movable] += rng.normal(0.0, scale, size=(len(movable), X.shape[1]))
    grid.global_nodes = X
    for bi, blk in enumerate(grid.blocks):
        blk.nodes[...] = X[grid.block_dof_maps[bi]]
    return X.copy()


def record(ref_root: Path) -> list[dict]:
    from oracle import oracle

    ref = oracle.load_ref("fp64snap")
    if ref is None:
        raise SystemExit("oracle/_ref/fp64snap missing: run oracle/build_ref.sh first")
    sys.path.insert(0, str(ref_root))
    sys.path.insert(0, str(ref_root / "examples" / "2D" / "circles"))
    import egg._cpp  # noqa: F401  (the package only; its compiled module is the proxy)

    rec = Recorder(ref)
    proxy = rec.module()
    sys.modules["egg._cpp.cpp_core"] = proxy
    sys.modules["egg._cpp"].cpp_core = proxy

    from topologies import build_circle_in_rectangle

    from egg.pipeline import _cpp_reduce
    from egg.smoothing.cpp_backend import (CppStructuredSweepSession, build_block_structured_context,
                                           cpp_structured_sweep, cpp_untangle)
    from egg.smoothing.solver import build_sweep_context
    from egg.smoothing.targets import IdentityTarget
    from egg.topology.builder import TopologyBuilder

    # 1. The 12-block circle-in-rectangle O-grid (singular fans): the
    #    one-shot structured sweep, reporting every 5 sweeps.
    rec.scenario = "ogrid_sweep"
    topo, _ = build_circle_in_rectangle(rough=False, R=1)
    grid = topo.initialize_grid()
    ctx = build_sweep_context(grid, IdentityTarget(d=topo.d))
    X0 = _perturb(grid, seed=3, scale=0.01)
    cpp_structured_sweep(ctx, grid, X0, 50, device="auto", report_every=5)

    # 2. Two conforming blocks through the driver's session wrapper: sweeps,
    #    shape+size, positions, FAS and its hierarchy.
    rec.scenario = "lr_session"
    b = TopologyBuilder(d=2)
    for name, pos in [("A", (0.0, 0.0)), ("D", (0.0, 2.0)), ("B", (2.0, 0.0)), ("C", (2.0, 2.0)),
                      ("E", (4.0, 0.0)), ("F", (4.0, 2.0))]:
        b.add_corner(name, pos, fixed=True)
    b.add_block("L", ("A", "D", "B", "C"), (16, 16))
    b.add_block("R", ("B", "C", "E", "F"), (16, 16))
    b.connect("L", 0, 1, "R", 0, 0)
    grid = b.build().initialize_grid()
    X0 = _perturb(grid, seed=5, scale=0.02)
    ctx = build_sweep_context(grid, IdentityTarget(2))
    s = CppStructuredSweepSession(ctx, build_block_structured_context(grid), X0, device="auto")
    s.run(20, report_every=1)
    s.run(10, phase="shape_size", omega=1.0, report_every=5)
    s._session.get_X()
    s.run_fas(3, omega=1.0)
    s._session.mg_levels()
    s._session.get_X()

    # 3. The delta-continuation untangle driver on a mildly folded O-grid
    #    (halfway between the valid and the rough initial grids).
    rec.scenario = "untangle"
    topo, _ = build_circle_in_rectangle(rough=True, R=3)
    grid = topo.initialize_grid()
    X_fold = grid.global_nodes.copy()
    X_ok = build_circle_in_rectangle(rough=False, R=3)[0].initialize_grid().global_nodes.copy()
    X0 = 0.5 * X_fold + 0.5 * X_ok
    grid.global_nodes = X0
    for bi, blk in enumerate(grid.blocks):
        blk.nodes[...] = X0[grid.block_dof_maps[bi]]
    ctx = build_sweep_context(grid, IdentityTarget(d=topo.d))
    cpp_untangle(ctx, grid, X0.copy(), device="auto", sweeps_per_delta=40, max_outer=60, margin=1e-9, omega=0.5)

    # 4. The pipeline's energy probe: one omega = 0 sweep as a reduction.
    rec.scenario = "pipeline_probe"
    topo, _ = build_circle_in_rectangle(rough=False, R=1)
    grid = topo.initialize_grid()
    ctx = build_sweep_context(grid, IdentityTarget(d=topo.d))
    _cpp_reduce(grid, ctx, "auto")
    _cpp_reduce(grid, ctx, "auto", phase="shape_size")
    return rec.events


TRACE_TOPO = HERE / "ref_dropin_topo.pkl.gz"


def record_topo(ref_root: Path) -> list[dict]:
    """``run_control_topo`` (``egg/smoothing/control_backend.py:646``) on the
    reference's own multi-block control test grids: a two-block seam with a
    wavy edge, a 2 x 2 crossing and a valence-3 fan, with C1 seams and fan
    penalty rows, plus a seam-orthogonality penalty run (per-iteration
    penalty uploads) and a C2-penalty run."""
    from oracle import oracle

    ref = oracle.load_ref("fp64snap")
    if ref is None:
        raise SystemExit("oracle/_ref/fp64snap missing: run oracle/build_ref.sh first")
    sys.path.insert(0, str(ref_root))
    import egg._cpp  # noqa: F401

    rec = Recorder(ref)
    proxy = rec.module()
    sys.modules["egg._cpp.cpp_core"] = proxy
    sys.modules["egg._cpp"].cpp_core = proxy

    from egg.smoothing.control_backend import run_control_topo
    from egg.smoothing.targets import IdentityTarget
    from tests.smoothing.test_control_topology import _fan_grid, _lr_grid, _perturb, _quad_grid

    exact = dict(pcg_forcing=False, pcg_rtol=1e-12, pcg_max_iter=2000)
    cases = [("seam", lambda: _lr_grid(wave=0.3), {}), ("crossing", _quad_grid, {}), ("fan", _fan_grid, {}),
             ("seam_c2", lambda: _lr_grid(wave=0.3), dict(c2_weight=0.5)),
             ("seam_ortho", lambda: _lr_grid(shear=0.3), dict(ortho="penalty", ortho_weight=1.0)),
             ("crossing_inexact", _quad_grid, dict(pcg_forcing=True, pcg_rtol=1e-10))]
    for name, make, kw in cases:
        rec.scenario = name
        grid = make()
        _perturb(grid)
        opts = dict(exact)
        opts.update(kw)
        run_control_topo(grid, IdentityTarget(2), device="auto", **opts)
    return rec.events


TRACE_WALLS = HERE / "ref_dropin_walls.pkl.gz"


def record_walls(ref_root: Path) -> list[dict]:
    """Single-block control nets with sliding walls, through the reference's
    own wall-session helpers (``tests/smoothing/test_control_wall_cpp.py``,
    wire ``egg/smoothing/control_backend.py:137-175``): an arc wall with the
    orthogonality dial off, a sheared arc wall in the three modes (off,
    penalty, hard) with exact PCG solves and once more in hard mode with the
    default inexact solves, and a 3D cube whose bottom face slides on a
    sphere (off and hard)."""
    from oracle import oracle

    ref = oracle.load_ref("fp64snap")
    if ref is None:
        raise SystemExit("oracle/_ref/fp64snap missing: run oracle/build_ref.sh first")
    sys.path.insert(0, str(ref_root))
    import egg._cpp  # noqa: F401

    rec = Recorder(ref)
    proxy = rec.module()
    sys.modules["egg._cpp.cpp_core"] = proxy
    sys.modules["egg._cpp"].cpp_core = proxy

    from tests.smoothing.test_control_wall import _make_arc_grid, _make_sheared_arc_grid
    from tests.smoothing.test_control_wall_cpp import (
        _make_sphere_cube_grid,
        _make_wall_session,
        _make_wall_session_3d,
    )

    def finish(sess):
        sess.get_C()
        sess.get_X()

    rec.scenario = "arc_off"
    grid, arc = _make_arc_grid()
    sess, _ = _make_wall_session(grid, arc, "off")
    sess.run_control(20)
    finish(sess)
    for ortho, weight in (("off", 0.0), ("penalty", 10.0), ("hard", 0.0)):
        rec.scenario = f"sheared_{ortho}"
        grid, arc = _make_sheared_arc_grid()
        sess, _ = _make_wall_session(grid, arc, ortho, weight=weight)
        sess.run_control(12, pcg_max_iter=500, pcg_rtol=1e-12, pcg_forcing=False)
        finish(sess)
    rec.scenario = "sheared_hard_inexact"
    grid, arc = _make_sheared_arc_grid()
    sess, _ = _make_wall_session(grid, arc, "hard")
    sess.run_control(25)
    finish(sess)
    for ortho in ("off", "hard"):
        rec.scenario = f"sphere_{ortho}"
        grid, sphere = _make_sphere_cube_grid()
        sess, _ = _make_wall_session_3d(grid, sphere, ortho)
        sess.run_control(10)
        finish(sess)
    return rec.events


TRACE_SLIDES = HERE / "ref_dropin_slides.pkl.gz"


def record_slides(ref_root: Path) -> list[dict]:
    """Topologies with sliding-wall frames and a 3D topology, through the
    reference's own tests of its multi-block driver
    (``tests/smoothing/test_control_topo_cpp.py``): a two-block seam whose
    bottom rides a line segment (then the same grid with fixed walls), a
    single block whose bottom rides a cubic B-spline, and a rotated 3D
    two-block slab.  Each test runs as written (its assertions check the
    reference core); the recorder keeps the calls."""
    from oracle import oracle

    ref = oracle.load_ref("fp64snap")
    if ref is None:
        raise SystemExit("oracle/_ref/fp64snap missing: run oracle/build_ref.sh first")
    sys.path.insert(0, str(ref_root))
    import egg._cpp  # noqa: F401

    rec = Recorder(ref)
    proxy = rec.module()
    sys.modules["egg._cpp.cpp_core"] = proxy
    sys.modules["egg._cpp"].cpp_core = proxy

    from tests.smoothing import test_control_topo_cpp as t

    for name, fn in (("line_seam", t.test_device_sliding_wall_roots),
                     ("bspline_block", t.test_single_block_segmented_wall),
                     ("slab3_rotated", t.test_device_3d_two_block_run)):
        rec.scenario = name
        fn()
    return rec.events


def _save(path: Path, events: list[dict]) -> None:
    with gzip.open(path, "wb") as f:
        pickle.dump({"events": events}, f, protocol=4)
    counts = {}
    for ev in events:
        counts[ev["scenario"]] = counts.get(ev["scenario"], 0) + 1
    print(f"{path.name}: {len(events)} calls {counts}")


if __name__ == "__main__":
    from oracle import oracle

    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    root = Path(args[0]) if args else oracle.reference_root()
    if root is None:
        raise SystemExit("reference checkout not found: pass its path or set EGG_REFERENCE_ROOT")
    if "--topo" in sys.argv:
        _save(TRACE_TOPO, record_topo(root))
    elif "--walls" in sys.argv:
        _save(TRACE_WALLS, record_walls(root))
    elif "--slides" in sys.argv:
        _save(TRACE_SLIDES, record_slides(root))
    else:
        _save(TRACE, record(root))
