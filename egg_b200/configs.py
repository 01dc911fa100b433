"""Seeded synthetic multi-block grids for the smoother workloads.

Every generator returns a :class:`Grid` (per-block global-id arrays, positions in
global node order, the moving-DOF mask).  Positions are built by transfinite
interpolation of straight/circular block edges and perturbed with
``numpy.random.default_rng(seed)``; nothing is read from disk.

* :func:`unit_square`   one n x n block on [0,1]^2, interior noise +-frac*h
  (the 4097^2 +-0.3h sweep workload and its small parity cases).
* :func:`disk_oh`       unit disk as a 5-block O-H grid: centre square of
  half-width 0.35 plus four curved blocks to the unit circle; circle fixed,
  every other node perturbed by +-frac * (local min edge length).
* :func:`tangled_square` n x n unit square with seeded interior nodes displaced
  by 0.8-1.5 h in random directions until a target fraction of cells holds an
  inverted corner sample (the untangling workload).
* :func:`unit_cube`     one n^3 block on [0,1]^3 with interior noise.
* :func:`sphere_in_cube` 7-block hex grid of the cube [-1,1]^3: a centre block
  mapped onto the ball r = 0.5 and six shell blocks from the sphere to the cube
  faces; cube boundary fixed, every other node perturbed by +-frac * (local min
  edge length).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import wire as _wire

__all__ = [
    "Grid", "unit_square", "disk_oh", "tangled_square", "unit_cube", "two_cubes", "sphere_in_cube",
    "grid_mindet", "mean_size_w_inv", "disk_on_curve", "square_sliding", "cube_sliding", "square_bezier",
    "cube_curved", "square_bspline", "square_composite",
]


@dataclass
class Grid:
    name: str
    d: int
    blocks: list[np.ndarray]
    X: np.ndarray  # (N, d) float64, global node order
    free: np.ndarray  # (N,) bool
    meta: dict = field(default_factory=dict)
    # constrained boundary nodes: global id -> (entity tag, record)
    constraints: dict = field(default_factory=dict)
    # soft terms: optional "directional" and "curvature" tables (wire.flat_wire)
    soft: dict = field(default_factory=dict)

    @property
    def num_nodes(self) -> int:
        return int(self.X.shape[0])

    @property
    def num_free(self) -> int:
        return int(self.free.sum())

    def wire(self, *, w_inv=None, compact: bool = False, device: str | None = None) -> dict:
        return _wire.flat_wire(self.blocks, self.free, self.d, w_inv=w_inv, compact=compact,
                               constraints=self.constraints, directional=self.soft.get("directional"),
                               curvature=self.soft.get("curvature"), device=device)

    def structured(self) -> dict:
        return _wire.structured_tables(self.blocks)

    def X_flat(self) -> np.ndarray:
        return np.ascontiguousarray(self.X, dtype=np.float64).ravel()


def _min_edge(blocks: list[np.ndarray], X: np.ndarray) -> np.ndarray:
    """Per-node minimum length of its incident block edges."""
    h = np.full(X.shape[0], np.inf)
    for ids in blocks:
        for ax in range(ids.ndim):
            a = np.take(ids, range(0, ids.shape[ax] - 1), axis=ax).reshape(-1)
            b = np.take(ids, range(1, ids.shape[ax]), axis=ax).reshape(-1)
            ln = np.linalg.norm(X[a] - X[b], axis=1)
            np.minimum.at(h, a, ln)
            np.minimum.at(h, b, ln)
    return h


def unit_square(n: int, frac: float = 0.3, seed: int = 0) -> Grid:
    """One n x n block on the unit square; node (i, j) at (i h, j h)."""
    ids = np.arange(n * n, dtype=np.int64).reshape(n, n)
    t = np.linspace(0.0, 1.0, n)
    X = np.stack(np.meshgrid(t, t, indexing="ij"), axis=-1).reshape(-1, 2).copy()
    free = np.zeros((n, n), dtype=bool)
    free[1:-1, 1:-1] = True
    free = free.reshape(-1)
    h = 1.0 / (n - 1)
    rng = np.random.default_rng(seed)
    if frac > 0:
        X[free] += rng.uniform(-frac * h, frac * h, size=(int(free.sum()), 2))
    return Grid(f"square{n}", 2, [ids], X, free, {"h": h, "frac": frac, "seed": seed})


def _dedupe(points: list[np.ndarray]):
    """Global ids for per-block point arrays, merging coincident nodes."""
    d = points[0].shape[-1]
    flat = np.concatenate([p.reshape(-1, d) for p in points])
    key = np.round(flat * 1e9).astype(np.int64)
    _, first, inv = np.unique(key, axis=0, return_index=True, return_inverse=True)
    # Ids in first-appearance order, so block 0 (the centre) numbers first.
    order = np.argsort(first, kind="stable")
    rank = np.empty_like(order)
    rank[order] = np.arange(order.size)
    gid = rank[inv.reshape(-1)]
    X = flat[np.sort(first)]
    blocks, off = [], 0
    for p in points:
        shp = p.shape[:-1]
        m = int(np.prod(shp))
        blocks.append(gid[off : off + m].reshape(shp))
        off += m
    return blocks, X


def disk_oh(n: int = 65, frac: float = 0.25, seed: int = 0, half_width: float = 0.35) -> Grid:
    """Unit disk, 5-block O-H topology, every block n x n nodes."""
    a = half_width
    s = np.linspace(-a, a, n)
    sq = np.stack(np.meshgrid(s, s, indexing="ij"), axis=-1)  # (n, n, 2): axis0 = x, axis1 = y
    u = np.linspace(0.0, 1.0, n)[:, None, None]
    pts = [sq]
    # Curved blocks: axis 0 radial (outward), axis 1 counter-clockwise.
    sides = [
        (np.stack([np.full(n, a), s], axis=1), -0.25 * np.pi),  # right
        (np.stack([s[::-1], np.full(n, a)], axis=1), 0.25 * np.pi),  # top
        (np.stack([np.full(n, -a), s[::-1]], axis=1), 0.75 * np.pi),  # left
        (np.stack([s, np.full(n, -a)], axis=1), 1.25 * np.pi),  # bottom
    ]
    for inner, th0 in sides:
        th = th0 + np.linspace(0.0, 0.5 * np.pi, n)
        outer = np.stack([np.cos(th), np.sin(th)], axis=1)
        pts.append((1.0 - u) * inner[None, :, :] + u * outer[None, :, :])
    blocks, X = _dedupe(pts)
    N = X.shape[0]
    free = np.ones(N, dtype=bool)
    for b in blocks[1:]:
        free[b[-1, :]] = False  # circle
    h = _min_edge(blocks, X)
    rng = np.random.default_rng(seed)
    noise = rng.uniform(-1.0, 1.0, size=(N, 2)) * (frac * h)[:, None]
    X = X + np.where(free[:, None], noise, 0.0)
    return Grid(f"disk_oh{n}", 2, blocks, X, free, {"frac": frac, "seed": seed, "half_width": a})


def disk_on_curve(n: int = 17, frac: float = 0.25, slide: float = 0.3, off: float = 0.02, seed: int = 0,
                  ry: float = 1.0, arcs: bool = False) -> Grid:
    """The 5-block O-H disk whose outer nodes slide on its boundary curve.

    ``ry == 1``: the unit circle (Circle entity, tag 2); with ``arcs`` each
    outer block's quarter of it instead (CircleArc entities, tag 6, open,
    angle ranges [-pi/4, pi/4], [pi/4, 3pi/4], [3pi/4, 5pi/4] (across the
    +-pi seam) and [-3pi/4, -pi/4]; a node shared by two blocks takes the
    first one's arc; with ``ry != 1`` EllipseArc quarters, tag 7, the last
    one [5pi/4, 7pi/4]).  Otherwise the disk is squeezed to the axis-aligned
    ellipse with semi-axes (1, ry) (Ellipse entity, tag 3).  Every boundary
    node is moved along the curve by up to ``slide`` of its spacing and off it
    by up to ``off`` of the local edge length, so the first sweep also
    projects.
    """
    g = disk_oh(n, frac=frac, seed=seed)
    X = g.X.copy()
    X[:, 1] *= ry
    bnd = np.flatnonzero(~g.free)
    rng = np.random.default_rng(seed + 101)
    h = _min_edge(g.blocks, X)
    th = np.arctan2(X[bnd, 1] / ry, X[bnd, 0])
    th += rng.uniform(-slide, slide, bnd.size) * (0.5 * np.pi / (n - 1))
    rad = 1.0 + rng.uniform(-off, off, bnd.size) * h[bnd]
    X[bnd, 0] = rad * np.cos(th)
    X[bnd, 1] = rad * ry * np.sin(th)
    tag, rec = (2, (0.0, 0.0, 1.0)) if ry == 1.0 else (3, (0.0, 0.0, 1.0, ry))
    cons = {int(b): (tag, rec) for b in bnd}
    kind = "circle" if tag == 2 else "ellipse"
    if arcs:
        cons = {}
        if ry == 1.0:  # CircleArc quarters
            starts = (-0.25 * np.pi, 0.25 * np.pi, 0.75 * np.pi, -0.75 * np.pi)
            ent = lambda t0: (6, (0.0, 0.0, 1.0, t0, t0 + 0.5 * np.pi, 0.0))
            kind = "arcs"
        else:  # EllipseArc quarters, parametric angle in [0, 2 pi) except the first
            starts = (-0.25 * np.pi, 0.25 * np.pi, 0.75 * np.pi, 1.25 * np.pi)
            ent = lambda t0: (7, (0.0, 0.0, 1.0, ry, 0.0, t0, t0 + 0.5 * np.pi, 0.0))
            kind = "earcs"
        for blk, t0 in zip(g.blocks[1:], starts):
            for v in blk[-1, :]:
                cons.setdefault(int(v), ent(t0))
    return Grid(f"disk_{kind}{n}", 2, g.blocks, X, g.free.copy(), {"frac": frac, "seed": seed, "ry": ry}, cons)


def square_sliding(n: int = 17, frac: float = 0.25, slide: float = 0.3, seed: int = 0,
                   rail_end: float = 0.6) -> Grid:
    """Unit square whose side nodes slide: three sides on LineSeg entities
    (tag 1), the top side on a LineRail (tag 15) from x = 0 to ``rail_end``,
    so top nodes beyond it are released and move freely.  Corners stay fixed.
    Side nodes move along their side by up to ``slide`` h; top nodes also sit
    up to 0.05 h off the line."""
    g = unit_square(n, frac=frac, seed=seed)
    ids = g.blocks[0]
    X = g.X.copy()
    h = 1.0 / (n - 1)
    rng = np.random.default_rng(seed + 202)
    cons = {}
    sides = [
        (ids[1:-1, 0], 0, (1, (0.0, 0.0, 1.0, 0.0))),           # bottom, y = 0: x slides
        (ids[-1, 1:-1], 1, (1, (1.0, 0.0, 1.0, 1.0))),          # right, x = 1: y slides
        (ids[0, 1:-1], 1, (1, (0.0, 0.0, 0.0, 1.0))),           # left, x = 0
        (ids[1:-1, -1], 0, (15, (0.0, 1.0, rail_end, 1.0))),    # top rail, y = 1
    ]
    for nodes, ax, ent in sides:
        X[nodes, ax] += rng.uniform(-slide, slide, nodes.size) * h
        if ent[0] == 15:
            X[nodes, 1 - ax] += rng.uniform(-0.05, 0.05, nodes.size) * h
        for v in nodes:
            cons[int(v)] = ent
    return Grid(f"square_slide{n}", 2, g.blocks, X, g.free.copy(),
                {"frac": frac, "seed": seed, "rail_end": rail_end}, cons)


def grid_mindet(blocks, X, d=2) -> np.ndarray:
    """det A of every canonical corner sample (energy-stencil order)."""
    _, gc, gn, sg = _wire.cell_stencil(blocks, d)
    cols = [sg[k][:, None] * (X[gn[k]] - X[gc]) for k in range(d)]
    if d == 2:
        return cols[0][:, 0] * cols[1][:, 1] - cols[1][:, 0] * cols[0][:, 1]
    return np.einsum("ij,ij->i", cols[0], np.cross(cols[1], cols[2]))


def tangled_square(n: int = 1025, target: float = 0.05, seed: int = 0, batch: int | None = None) -> Grid:
    """n x n unit square with ~``target`` of cells inverted by node displacements."""
    g = unit_square(n, frac=0.0, seed=seed)
    h = 1.0 / (n - 1)
    rng = np.random.default_rng(seed)
    X = g.X.copy()
    interior = np.flatnonzero(g.free)
    order = rng.permutation(interior)
    ncell = (n - 1) ** 2
    batch = batch or max(1, ncell // 400)
    used = 0
    frac_bad = 0.0
    while frac_bad < target and used < order.size:
        pick = order[used : used + batch]
        used += pick.size
        r = rng.uniform(0.8, 1.5, size=pick.size) * h
        th = rng.uniform(0.0, 2.0 * np.pi, size=pick.size)
        X[pick, 0] += r * np.cos(th)
        X[pick, 1] += r * np.sin(th)
        det = grid_mindet(g.blocks, X).reshape(ncell, 4)
        frac_bad = float((det <= 0).any(axis=1).mean())
    return Grid(
        f"tangled{n}", 2, g.blocks, X, g.free,
        {"h": h, "seed": seed, "displaced": int(used), "inverted_cell_fraction": frac_bad},
    )


def mean_size_w_inv(blocks, X, d=2) -> np.ndarray:
    """Inverse of the mean-size target W = hbar I (det W = mean det A)."""
    vol = abs(float(grid_mindet(blocks, X, d).mean()))
    hbar = vol ** (1.0 / d)
    return np.eye(d) / hbar


def unit_cube(n: int, frac: float = 0.2, seed: int = 0) -> Grid:
    """One n^3 block on the unit cube; node (i, j, k) at (i h, j h, k h)."""
    ids = np.arange(n**3, dtype=np.int64).reshape(n, n, n)
    t = np.linspace(0.0, 1.0, n)
    X = np.stack(np.meshgrid(t, t, t, indexing="ij"), axis=-1).reshape(-1, 3).copy()
    free = np.zeros((n, n, n), dtype=bool)
    free[1:-1, 1:-1, 1:-1] = True
    free = free.reshape(-1)
    h = 1.0 / (n - 1)
    rng = np.random.default_rng(seed)
    if frac > 0:
        X[free] += rng.uniform(-frac * h, frac * h, size=(int(free.sum()), 3))
    return Grid(f"cube{n}", 3, [ids], X, free, {"h": h, "frac": frac, "seed": seed})


def _bezier(P: np.ndarray, t: np.ndarray) -> np.ndarray:
    n = len(P) - 1
    from math import comb

    return sum(comb(n, i) * ((1 - t) ** (n - i) * t**i)[:, None] * P[i] for i in range(n + 1))


def square_bezier(n: int = 17, frac: float = 0.2, slide: float = 0.3, seed: int = 0) -> Grid:
    """Unit square whose bottom side bends into the quadratic Bezier
    (0,0)-(0.5,-0.12)-(1,0) (QuadBezier, tag 8) and whose top side into the
    cubic (0,1)-(0.3,1.15)-(0.7,0.9)-(1,1) (CubicBezier, tag 9), both trimmed
    to [0, 1]; their nodes sit on the curves at parameters i/(n-1), moved by up
    to ``slide`` of a step, and slide along them.  Corners stay fixed."""
    g = unit_square(n, frac=frac, seed=seed)
    ids = g.blocks[0]
    X = g.X.copy()
    rng = np.random.default_rng(seed + 404)
    t = np.linspace(0.0, 1.0, n)[1:-1] + rng.uniform(-slide, slide, n - 2) / (n - 1)
    quad = np.array([[0.0, 0.0], [0.5, -0.12], [1.0, 0.0]])
    cub = np.array([[0.0, 1.0], [0.3, 1.15], [0.7, 0.9], [1.0, 1.0]])
    cons = {}
    for nodes, P, tag in ((ids[1:-1, 0], quad, 8), (ids[1:-1, -1], cub, 9)):
        X[nodes] = _bezier(P, t)
        rec = tuple(float(x) for x in P.ravel()) + (0.0, 1.0)
        for v in nodes:
            cons[int(v)] = (tag, rec)
    return Grid(f"square_bezier{n}", 2, g.blocks, X, g.free.copy(), {"frac": frac, "seed": seed}, cons)


def _nurbs_points(deg, knots, ctrl, w, t):
    from scipy.interpolate import BSpline

    ctrl = np.asarray(ctrl, dtype=np.float64)
    w = np.ones(len(ctrl)) if w is None else np.asarray(w, dtype=np.float64)
    num = BSpline(np.asarray(knots), ctrl * w[:, None], deg)(t)
    den = BSpline(np.asarray(knots), w, deg)(t)
    return num / den[:, None]


def square_bspline(n: int = 17, frac: float = 0.2, slide: float = 0.3, seed: int = 0) -> Grid:
    """Unit square whose top side is a clamped cubic B-spline through six
    control points and whose bottom side is a rational quadratic NURBS
    (B-spline entities, tag 10, trimmed to [0, 1]); their nodes sit on the
    curves at parameters i/(n-1), moved by up to ``slide`` of a step, and
    slide along them.  Corners stay fixed."""
    g = unit_square(n, frac=frac, seed=seed)
    ids = g.blocks[0]
    X = g.X.copy()
    rng = np.random.default_rng(seed + 606)
    t = np.linspace(0.0, 1.0, n)[1:-1] + rng.uniform(-slide, slide, n - 2) / (n - 1)
    top = (3, [0, 0, 0, 0, 1 / 3, 2 / 3, 1, 1, 1, 1],
           [[0, 1], [0.2, 1.1], [0.4, 0.95], [0.6, 1.08], [0.8, 0.97], [1, 1]], None)
    bot = (2, [0, 0, 0, 0.5, 1, 1, 1], [[0, 0], [0.3, -0.12], [0.7, -0.08], [1, 0]], [1.0, 0.8, 1.2, 1.0])
    cons = {}
    for nodes, (deg, knots, ctrl, w) in ((ids[1:-1, -1], top), (ids[1:-1, 0], bot)):
        X[nodes] = _nurbs_points(deg, knots, ctrl, w, t)
        rec = (float(deg), float(len(ctrl)), 0.0, 1.0, 0.0, 0.0 if w is None else 1.0)
        seg = (np.asarray(knots, dtype=np.float64), np.asarray(ctrl, dtype=np.float64).ravel(),
               np.zeros(0) if w is None else np.asarray(w, dtype=np.float64))
        for v in nodes:
            cons[int(v)] = (10, rec, seg)
    return Grid(f"square_bspline{n}", 2, g.blocks, X, g.free.copy(), {"frac": frac, "seed": seed}, cons)


def _composite_block(segs) -> np.ndarray:
    """Composite segment records: [tag, params...] padded to 13 reals each."""
    out = np.zeros((len(segs), 13))
    for k, (tag, params) in enumerate(segs):
        out[k, 0] = tag
        out[k, 1 : 1 + len(params)] = params
    return out.ravel()


def square_composite(n: int = 17, frac: float = 0.2, slide: float = 0.3, seed: int = 0) -> Grid:
    """Unit square whose bottom and top sides are composite paths (tag 11):
    bottom = LineSeg (0,0)-(0.3,0), QuadBezier (0.3,0)-(0.5,-0.05)-(0.7,0),
    LineSeg (0.7,0)-(1,0); top = CubicBezier (0,1)-(0.2,1.05)-(0.4,1.03)-(0.5,1)
    then a shallow arc of the ellipse about (0.75, 1.27) with semi-axes
    (0.25 / sqrt(0.19), 0.3) from (0.5, 1) to (1, 1) (EllipseArc).  Side nodes sit on their
    path at x = i/(n-1) moved by up to ``slide`` of a step, and slide along
    it.  Corners stay fixed."""
    g = unit_square(n, frac=frac, seed=seed)
    ids = g.blocks[0]
    X = g.X.copy()
    rng = np.random.default_rng(seed + 707)
    x = np.linspace(0.0, 1.0, n)[1:-1] + rng.uniform(-slide, slide, n - 2) / (n - 1)
    bot = [(1, (0.0, 0.0, 0.3, 0.0)), (8, (0.3, 0.0, 0.5, -0.05, 0.7, 0.0, 0.0, 1.0)), (1, (0.7, 0.0, 1.0, 0.0))]
    ea = 0.25 / np.sqrt(0.19)
    t0, t1 = np.arctan2(-0.9, -0.25 / ea) % (2 * np.pi), np.arctan2(-0.9, 0.25 / ea) % (2 * np.pi)
    top = [(9, (0.0, 1.0, 0.2, 1.05, 0.4, 1.03, 0.5, 1.0, 0.0, 1.0)),
           (7, (0.75, 1.27, ea, 0.3, 0.0, t0, t1, 0.0))]
    yb = np.where((x > 0.3) & (x < 0.7), 2 * (1 - (x - 0.3) / 0.4) * ((x - 0.3) / 0.4) * -0.05, 0.0)
    X[ids[1:-1, 0]] = np.stack([x, yb], axis=1)
    tt = np.clip(x / 0.5, 0.0, 1.0)
    cub = _bezier(np.array(top[0][1][:8]).reshape(4, 2), tt)
    ang = t0 + (t1 - t0) * np.clip((x - 0.5) / 0.5, 0.0, 1.0)
    ell = np.stack([0.75 + ea * np.cos(ang), 1.27 + 0.3 * np.sin(ang)], axis=1)
    X[ids[1:-1, -1]] = np.where((x <= 0.5)[:, None], cub, ell)
    cons = {}
    for nodes, segs in ((ids[1:-1, 0], bot), (ids[1:-1, -1], top)):
        blk = _composite_block(segs)
        for v in nodes:
            cons[int(v)] = (11, (float(len(segs)), 0.0), (blk,))
    return Grid(f"square_composite{n}", 2, g.blocks, X, g.free.copy(), {"frac": frac, "seed": seed}, cons)


def _composite_slice(segs) -> np.ndarray:
    """A composite path's arena slice: the segment records ([tag, params...]
    padded to 13 reals) followed by each B-spline segment's knots, control
    points and weights.  A B-spline segment is given as
    ``(10, (degree, knots, ctrl, weights or None, t0, t1))`` and its record
    blob becomes [degree, n_ctrl, knot_off, ctrl_off, t0, t1, w_off, has_w]
    with offsets into the slice (``src/geometry.hpp:1524-1550``)."""
    recs = np.zeros((len(segs), 13))
    data: list[np.ndarray] = []
    at = recs.size
    for k, (tag, params) in enumerate(segs):
        recs[k, 0] = tag
        if tag != 10:
            recs[k, 1 : 1 + len(params)] = params
            continue
        deg, knots, ctrl, w, t0, t1 = params
        knots = np.asarray(knots, dtype=np.float64)
        ctrl = np.asarray(ctrl, dtype=np.float64).ravel()
        ko, co = at, at + knots.size
        at = co + ctrl.size
        data += [knots, ctrl]
        wo = at
        if w is not None:
            data.append(np.asarray(w, dtype=np.float64))
            at += len(w)
        recs[k, 1:9] = (deg, ctrl.size // 2, ko, co, t0, t1, wo, 0.0 if w is None else 1.0)
    return np.concatenate([recs.ravel()] + data)


def square_composite_bspline(n: int = 17, frac: float = 0.2, slide: float = 0.3, seed: int = 0) -> Grid:
    """Unit square whose bottom and top sides are composite paths with
    B-spline segments: bottom = LineSeg (0,0)-(0.3,0), a clamped cubic
    B-spline from (0.3,0) to (0.7,0) dipping below the side, LineSeg
    (0.7,0)-(1,0); top = a rational quadratic NURBS from (0,1) to (0.6,1),
    then LineSeg (0.6,1)-(1,1).  Side nodes sit on their path (on the
    spline at the parameter their x maps to), moved by up to ``slide`` of a
    step, and slide along it.  Corners stay fixed."""
    g = unit_square(n, frac=frac, seed=seed)
    ids = g.blocks[0]
    X = g.X.copy()
    rng = np.random.default_rng(seed + 808)
    x = np.linspace(0.0, 1.0, n)[1:-1] + rng.uniform(-slide, slide, n - 2) / (n - 1)
    b_sp = (3, [0, 0, 0, 0, 0.5, 1, 1, 1, 1], [[0.3, 0], [0.4, -0.06], [0.5, 0.02], [0.6, -0.05], [0.7, 0]], None,
            0.0, 1.0)
    t_sp = (2, [0, 0, 0, 1 / 3, 2 / 3, 1, 1, 1], [[0, 1], [0.15, 1.06], [0.3, 0.98], [0.45, 1.04], [0.6, 1]],
            [1.0, 0.8, 1.2, 0.9, 1.0], 0.0, 1.0)
    bot = [(1, (0.0, 0.0, 0.3, 0.0)), (10, b_sp), (1, (0.7, 0.0, 1.0, 0.0))]
    top = [(10, t_sp), (1, (0.6, 1.0, 1.0, 1.0))]
    tb = np.clip((x - 0.3) / 0.4, 0.0, 1.0)
    pb = _nurbs_points(b_sp[0], b_sp[1], b_sp[2], b_sp[3], tb)
    X[ids[1:-1, 0]] = np.where(((x > 0.3) & (x < 0.7))[:, None], pb, np.stack([x, np.zeros_like(x)], axis=1))
    tt = np.clip(x / 0.6, 0.0, 1.0)
    pt = _nurbs_points(t_sp[0], t_sp[1], t_sp[2], t_sp[3], tt)
    X[ids[1:-1, -1]] = np.where((x < 0.6)[:, None], pt, np.stack([x, np.ones_like(x)], axis=1))
    cons = {}
    for nodes, segs in ((ids[1:-1, 0], bot), (ids[1:-1, -1], top)):
        sl = _composite_slice(segs)
        for v in nodes:
            cons[int(v)] = (11, (float(len(segs)), 0.0), (sl,))
    return Grid(f"square_compbsp{n}", 2, g.blocks, X, g.free.copy(), {"frac": frac, "seed": seed}, cons)


def cube_sliding(n: int = 9, frac: float = 0.2, slide: float = 0.3, off: float = 0.02, seed: int = 0,
                 rail_end: float = 0.6) -> Grid:
    """Unit cube whose face nodes slide on their planes (Plane entities, tag 5)
    on four faces: x = 0, x = 1, y = 0, and z = 1 with in-plane axes rotated
    by 0.3 rad.  The nodes of the edge y = z = 0 slide on a LineRail3 (tag 16)
    from x = 0 to ``rail_end``, so those beyond it are released.  The faces
    y = 1 and z = 0 and the other edges stay fixed.  Face and edge nodes move
    along their entity by up to ``slide`` h and off it by up to ``off`` h."""
    g = unit_cube(n, frac=frac, seed=seed)
    ids = g.blocks[0]
    X = g.X.copy()
    h = 1.0 / (n - 1)
    rng = np.random.default_rng(seed + 303)
    c, sn = np.cos(0.3), np.sin(0.3)
    inner = slice(1, -1)
    faces = [
        (ids[0, inner, inner], 0, (0.0, 0, 0, 0, 1, 0, 0, 0, 1)),
        (ids[-1, inner, inner], 0, (1.0, 0, 0, 0, 1, 0, 0, 0, 1)),
        (ids[inner, 0, inner], 1, (0.0, 0, 0, 1, 0, 0, 0, 0, 1)),
        (ids[inner, inner, -1], 2, (0.0, 0, 1, c, sn, 0, -sn, c, 0)),
    ]
    cons = {}
    for nodes, normal, rec in faces:
        nodes = nodes.reshape(-1)
        for ax in range(3):
            amp = off if ax == normal else slide
            X[nodes, ax] += rng.uniform(-amp, amp, nodes.size) * h
        for v in nodes:
            cons[int(v)] = (5, tuple(float(x) for x in rec))
    edge = ids[inner, 0, 0].reshape(-1)
    X[edge, 0] += rng.uniform(-slide, slide, edge.size) * h
    X[edge, 1:] += rng.uniform(-off, off, (edge.size, 2)) * h
    for v in edge:
        cons[int(v)] = (16, (0.0, 0.0, 0.0, rail_end, 0.0, 0.0))
    return Grid(f"cube_slide{n}", 3, g.blocks, X, g.free.copy(), {"frac": frac, "seed": seed}, cons)


def cube_curved(n: int = 9, frac: float = 0.15, slide: float = 0.3, off: float = 0.02, seed: int = 0) -> Grid:
    """Unit cube with curved faces whose nodes slide on them: the top face on
    the sphere of radius 4 about (0.5, 0.5, -3) (Sphere, tag 4), the face
    x ~ 1 on the cylinder of radius 4 about the z-parallel axis through
    (-3, 0.5) (Cylinder, tag 12), the face y = 0 on its plane (Plane, tag 5),
    and the edge y = z = 0 on the line x in [0.05, 0.95] (Line3, tag 13).  The
    other faces and edges stay fixed.  Nodes move along their entity by up to
    ``slide`` h and off it by up to ``off`` h."""
    g = unit_cube(n, frac=frac, seed=seed)
    ids = g.blocks[0]
    X = g.X.copy()
    h = 1.0 / (n - 1)
    rng = np.random.default_rng(seed + 505)
    inner = slice(1, -1)
    cons = {}
    # cylinder face: x from the cylinder at (y, z)
    cyl = ids[-1, inner, inner].reshape(-1)
    X[cyl, 1:] += rng.uniform(-slide, slide, (cyl.size, 2)) * h
    X[cyl, 0] = -3.0 + np.sqrt(16.0 - (X[cyl, 1] - 0.5) ** 2) + rng.uniform(-off, off, cyl.size) * h
    for v in cyl:
        cons[int(v)] = (12, (-3.0, 0.5, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 4.0))
    # sphere cap: z from the sphere at (x, y)
    sph = ids[inner, inner, -1].reshape(-1)
    X[sph, :2] += rng.uniform(-slide, slide, (sph.size, 2)) * h
    X[sph, 2] = -3.0 + np.sqrt(16.0 - (X[sph, 0] - 0.5) ** 2 - (X[sph, 1] - 0.5) ** 2)
    X[sph, 2] += rng.uniform(-off, off, sph.size) * h
    for v in sph:
        # chart frame ax = x, ay = z (pole along -y): the cap lies on the chart's
        # equator, away from the latitude's ill-conditioned poles
        cons[int(v)] = (4, (0.5, 0.5, -3.0, 4.0, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0))
    # plane face y = 0
    pl = ids[inner, 0, inner].reshape(-1)
    X[pl, 0] += rng.uniform(-slide, slide, pl.size) * h
    X[pl, 2] += rng.uniform(-slide, slide, pl.size) * h
    X[pl, 1] += rng.uniform(-off, off, pl.size) * h
    for v in pl:
        cons[int(v)] = (5, (0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0))
    # edge line y = z = 0, trimmed
    ed = ids[inner, 0, 0].reshape(-1)
    X[ed, 0] += rng.uniform(-slide, slide, ed.size) * h
    X[ed, 1:] += rng.uniform(-off, off, (ed.size, 2)) * h
    for v in ed:
        cons[int(v)] = (13, (0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.05, 0.95))
    return Grid(f"cube_curved{n}", 3, g.blocks, X, g.free.copy(), {"frac": frac, "seed": seed}, cons)


def _bsurf_points(pu, pv, ku, kv, ctrl, w, u, v):
    """Points of a tensor-product B-spline / NURBS surface at (u[i], v[i])."""
    from scipy.interpolate import BSpline

    ctrl = np.asarray(ctrl, dtype=np.float64)
    nu, nv = ctrl.shape[:2]
    w = np.ones((nu, nv)) if w is None else np.asarray(w, dtype=np.float64).reshape(nu, nv)
    Nu = BSpline.design_matrix(np.asarray(u), np.asarray(ku, dtype=np.float64), pu).toarray()
    Nv = BSpline.design_matrix(np.asarray(v), np.asarray(kv, dtype=np.float64), pv).toarray()
    num = np.einsum("pi,pj,ijc->pc", Nu, Nv, ctrl * w[..., None])
    den = np.einsum("pi,pj,ij->p", Nu, Nv, w)
    return num / den[:, None]


def _bsurf_entity(pu, pv, ku, kv, ctrl, w=None, trim=None):
    """(tag, record, seg) of a B-spline surface in the wire's SoA form
    (tag 14: (pu, pv, nu, nv, 0, 0, 0, 0, has_w) and the knots_u, knots_v,
    control net, weights, trim vertices and trim loop offsets fields)."""
    ctrl = np.asarray(ctrl, dtype=np.float64)
    nu, nv = ctrl.shape[:2]
    rec = (float(pu), float(pv), float(nu), float(nv), 0.0, 0.0, 0.0, 0.0, 0.0 if w is None else 1.0)
    verts = np.zeros(0) if trim is None else np.concatenate([np.asarray(lp, float).ravel() for lp in trim])
    loops = np.zeros(0) if trim is None else np.concatenate([[0], np.cumsum([len(lp) for lp in trim])]).astype(float)
    seg = (np.asarray(ku, dtype=np.float64), np.asarray(kv, dtype=np.float64), ctrl.reshape(-1),
           np.zeros(0) if w is None else np.asarray(w, dtype=np.float64).reshape(-1), verts, loops)
    return 14, rec, seg


# The two surfaces of cube_bsurf: a bicubic bump over the top face and a
# rational biquadratic (NURBS) sheet over the face x ~ 1, each spanning its
# face with a margin.
BSURF_TOP = dict(pu=3, pv=3, ku=[0, 0, 0, 0, 0.5, 1, 1, 1, 1], kv=[0, 0, 0, 0, 0.5, 1, 1, 1, 1])
BSURF_SIDE = dict(pu=2, pv=2, ku=[0, 0, 0, 0.5, 1, 1, 1], kv=[0, 0, 0, 0.5, 1, 1, 1])


def bsurf_nets():
    g = np.linspace(-0.1, 1.1, 5)
    top = np.zeros((5, 5, 3))
    top[..., 0], top[..., 1] = np.meshgrid(g, g, indexing="ij")
    bump = np.array([[0.0, 0.01, 0.02, 0.01, 0.0], [0.01, 0.05, 0.07, 0.04, 0.0], [0.02, 0.06, 0.1, 0.06, 0.02],
                     [0.0, 0.03, 0.05, 0.04, 0.01], [0.0, 0.0, 0.02, 0.01, 0.0]])
    top[..., 2] = 1.0 + bump
    h = np.linspace(-0.1, 1.1, 4)
    side = np.zeros((4, 4, 3))
    side[..., 1], side[..., 2] = np.meshgrid(h, h, indexing="ij")
    side[..., 0] = 1.0 + np.array([[0.0, 0.02, 0.02, 0.0], [0.01, 0.05, 0.04, 0.0],
                                   [0.0, 0.04, 0.06, 0.01], [0.0, 0.0, 0.01, 0.0]])
    w = np.array([[1.0, 0.9, 1.1, 1.0], [1.0, 1.2, 0.8, 1.0], [1.0, 0.85, 1.15, 1.0], [1.0, 1.0, 1.0, 1.0]])
    return top, side, w


def cube_bsurf(n: int = 9, frac: float = 0.15, slide: float = 0.3, off: float = 0.02, seed: int = 0) -> Grid:
    """Unit cube whose top face slides on a bicubic B-spline surface (a bump
    of up to 0.1 over z = 1) and whose face x ~ 1 slides on a rational
    biquadratic NURBS sheet (B-spline surfaces, tag 14).  Face nodes sit on
    the surfaces near their grid positions, moved along them by up to
    ``slide`` h and off them by up to ``off`` h; the other faces and all edges
    stay fixed."""
    g = unit_cube(n, frac=frac, seed=seed)
    ids = g.blocks[0]
    X = g.X.copy()
    h = 1.0 / (n - 1)
    rng = np.random.default_rng(seed + 707)
    inner = slice(1, -1)
    top, side, w = bsurf_nets()
    cons = {}
    t = BSURF_TOP
    nodes = ids[inner, inner, -1].reshape(-1)
    uv = (X[nodes, :2] + 0.1) / 1.2 + rng.uniform(-slide, slide, (nodes.size, 2)) * h / 1.2
    X[nodes] = _bsurf_points(t["pu"], t["pv"], t["ku"], t["kv"], top, None, uv[:, 0], uv[:, 1])
    X[nodes, 2] += rng.uniform(-off, off, nodes.size) * h
    ent = _bsurf_entity(t["pu"], t["pv"], t["ku"], t["kv"], top)
    for v in nodes:
        cons[int(v)] = ent
    t = BSURF_SIDE
    nodes = ids[-1, inner, inner].reshape(-1)
    uv = (X[nodes, 1:] + 0.1) / 1.2 + rng.uniform(-slide, slide, (nodes.size, 2)) * h / 1.2
    X[nodes] = _bsurf_points(t["pu"], t["pv"], t["ku"], t["kv"], side, w, uv[:, 0], uv[:, 1])
    X[nodes, 0] += rng.uniform(-off, off, nodes.size) * h
    ent = _bsurf_entity(t["pu"], t["pv"], t["ku"], t["kv"], side, w)
    for v in nodes:
        cons[int(v)] = ent
    return Grid(f"cube_bsurf{n}", 3, g.blocks, X, g.free.copy(), {"frac": frac, "seed": seed}, cons)


def two_cubes(n: int, frac: float = 0.2, seed: int = 0) -> Grid:
    """Two n^3 unit cubes sharing the x = 1 face (conforming 3D interface)."""
    t = np.linspace(0.0, 1.0, n)
    P = np.stack(np.meshgrid(t, t, t, indexing="ij"), axis=-1)
    blocks, X = _dedupe([P, P + np.array([1.0, 0.0, 0.0])])
    free = np.ones(X.shape[0], dtype=bool)
    for b in blocks:
        for ax in range(3):
            for side in (0, -1):
                face = np.take(b, side, axis=ax)
                if not (ax == 0 and ((b is blocks[0] and side == -1) or (b is blocks[1] and side == 0))):
                    free[face.reshape(-1)] = False
    h = 1.0 / (n - 1)
    rng = np.random.default_rng(seed)
    noise = rng.uniform(-frac * h, frac * h, size=X.shape)
    X = X + np.where(free[:, None], noise, 0.0)
    return Grid(f"two_cubes{n}", 3, blocks, X, free, {"h": h, "frac": frac, "seed": seed})


# Shell blocks: outward normal n and tangents t1, t2 with n x t1 = t2, so each
# block's (radial, t1, t2) logical axes are right-handed.
_SHELLS = [
    ((1, 0, 0), (0, 1, 0), (0, 0, 1)),
    ((-1, 0, 0), (0, 0, 1), (0, 1, 0)),
    ((0, 1, 0), (0, 0, 1), (1, 0, 0)),
    ((0, -1, 0), (1, 0, 0), (0, 0, 1)),
    ((0, 0, 1), (1, 0, 0), (0, 1, 0)),
    ((0, 0, -1), (0, 1, 0), (1, 0, 0)),
]


def sphere_in_cube(n: int = 129, frac: float = 0.2, seed: int = 0, radius: float = 0.5,
                   core: float = 0.25) -> Grid:
    """7-block sphere-in-cube hex grid of [-1,1]^3, every block n^3 nodes.

    Centre block: the cube [-core, core]^3.  Shell block with outward normal
    n: along its radial axis a node moves from the centre cube's face (r = 0)
    through the sphere of ``radius`` (r = 1/2, a node layer when n is odd) to
    the outer cube face (r = 1), piecewise linearly; its other two axes follow
    the face tangents.  Every block corner keeps three non-coplanar edges.
    """
    u = np.linspace(-1.0, 1.0, n)
    P = np.stack(np.meshgrid(u, u, u, indexing="ij"), axis=-1)
    pts = [core * P]
    r = np.linspace(0.0, 1.0, n)[:, None, None, None]
    for nrm, t1, t2 in _SHELLS:
        nrm, t1, t2 = (np.asarray(v, dtype=np.float64) for v in (nrm, t1, t2))
        V, W = np.meshgrid(u, u, indexing="ij")
        d = nrm[None, None, :] + V[..., None] * t1[None, None, :] + W[..., None] * t2[None, None, :]
        inner = core * d
        sph = radius * d / np.linalg.norm(d, axis=-1, keepdims=True)
        lo = inner[None] + np.minimum(2.0 * r, 1.0) * (sph - inner)[None]
        x = np.where(r <= 0.5, lo, sph[None] + (2.0 * r - 1.0) * (d - sph)[None])
        pts.append(x)
    blocks, X = _dedupe(pts)
    N = X.shape[0]
    free = np.ones(N, dtype=bool)
    for b in blocks[1:]:
        free[b[-1]] = False  # outer cube faces
    h = _min_edge(blocks, X)
    rng = np.random.default_rng(seed)
    noise = rng.uniform(-1.0, 1.0, size=(N, 3)) * (frac * h)[:, None]
    X = X + np.where(free[:, None], noise, 0.0)
    return Grid(f"sphere_in_cube{n}", 3, blocks, X, free, {"frac": frac, "seed": seed, "radius": radius})


def _log_uniform_odd(rng, lo: int, hi: int) -> int:
    n = int(round(float(np.exp(rng.uniform(np.log(lo), np.log(hi))))))
    n += 1 - n % 2
    return int(min(max(n, lo), hi))


def multiblock_mesh(seed: int, *, min_blocks: int = 3, max_blocks: int = 9, lo: int = 17, hi: int = 257,
                    frac: float = 0.25) -> Grid:
    """A conforming 2D multi-block mesh: a random 4-connected set of
    `min_blocks..max_blocks` cells of an r x c arrangement of rectangles
    (strips, L, T and zig-zag shapes arise), every row of cells sharing one
    node count in y and every column one in x, counts log-uniform odd in
    [lo, hi].  Uniform spacing h = 1 / (hi - 1); nodes on the outline of the
    union are fixed, every other node carries seeded uniform noise of
    +-frac h."""
    rng = np.random.default_rng(seed)
    nb = int(rng.integers(min_blocks, max_blocks + 1))
    while True:
        r, c = int(rng.integers(1, 4)), int(rng.integers(1, 10))
        if r * c >= nb:
            break
    cells = [(int(rng.integers(r)), int(rng.integers(c)))]
    steps = ((1, 0), (-1, 0), (0, 1), (0, -1))
    while len(cells) < nb:
        i, j = cells[int(rng.integers(len(cells)))]
        di, dj = steps[int(rng.integers(4))]
        cand = (i + di, j + dj)
        if 0 <= cand[0] < r and 0 <= cand[1] < c and cand not in cells:
            cells.append(cand)
    cells.sort()
    ny = [_log_uniform_odd(rng, lo, hi) for _ in range(r)]
    nx = [_log_uniform_odd(rng, lo, hi) for _ in range(c)]
    h = 1.0 / (hi - 1)
    y0 = np.concatenate([[0.0], np.cumsum([(n - 1) * h for n in ny])])
    x0 = np.concatenate([[0.0], np.cumsum([(n - 1) * h for n in nx])])
    pts = []
    for i, j in cells:
        xs = x0[j] + h * np.arange(nx[j])
        ys = y0[i] + h * np.arange(ny[i])
        pts.append(np.stack(np.meshgrid(xs, ys, indexing="ij"), axis=-1))
    blocks, X = _dedupe(pts)
    # Outline: block-side edges that belong to one block only.
    count: dict[tuple[int, int], int] = {}
    for b in blocks:
        for side in (b[0, :], b[-1, :], b[:, 0], b[:, -1]):
            for u, v in zip(side[:-1], side[1:]):
                e = (int(min(u, v)), int(max(u, v)))
                count[e] = count.get(e, 0) + 1
    fixed = np.zeros(X.shape[0], dtype=bool)
    for (u, v), k in count.items():
        if k == 1:
            fixed[u] = fixed[v] = True
    free = ~fixed
    X = X.copy()
    X[free] += rng.uniform(-frac * h, frac * h, size=(int(free.sum()), 2))
    return Grid(f"mb{seed}", 2, blocks, X, free,
                {"h": h, "frac": frac, "seed": seed, "cells": cells, "nx": nx, "ny": ny})


def batch_meshes(n_meshes: int = 256, seed: int = 0, **kw) -> list[Grid]:
    """Independent multi-block meshes for the batched sweep (mesh k uses seed
    seed * 100003 + k)."""
    return [multiblock_mesh(seed * 100003 + k, **kw) for k in range(n_meshes)]


def two_squares(n_big: int = 17, n_small: int = 6, frac: float = 0.2, seed: int = 0) -> Grid:
    """Two separate square blocks in one grid: [0, 4]^2 with n_big^2 nodes and
    [6, 8] x [0, 2] with n_small^2 nodes (an even count cannot coarsen by 2).
    Boundary nodes fixed, interior nodes carry seeded +-frac h noise."""
    rng = np.random.default_rng(seed)
    Xs, blocks, frees, off = [], [], [], 0
    for n, x0, side in ((n_big, 0.0, 4.0), (n_small, 6.0, 2.0)):
        t = np.linspace(0.0, side, n)
        X = np.stack(np.meshgrid(t, t, indexing="ij"), axis=-1).reshape(-1, 2)
        X[:, 0] += x0
        free = np.zeros((n, n), dtype=bool)
        free[1:-1, 1:-1] = True
        free = free.reshape(-1)
        h = side / (n - 1)
        X[free] += rng.uniform(-frac * h, frac * h, size=(int(free.sum()), 2))
        Xs.append(X)
        frees.append(free)
        blocks.append(off + np.arange(n * n, dtype=np.int64).reshape(n, n))
        off += n * n
    return Grid(f"two_squares{n_big}_{n_small}", 2, blocks, np.concatenate(Xs), np.concatenate(frees),
                {"frac": frac, "seed": seed})


def with_soft_terms(g: Grid, seed: int = 0, *, n_dir: int = 36, n_curv: int = 24, weight: float = 0.3,
                    block: int = 0) -> Grid:
    """Attaches seeded soft terms to a grid, on grid lines of one block:
    directional samples of every kind (parallel: two consecutive nodes, ref
    the unit normal of their initial segment, tilted; line: three
    consecutive nodes; stem: a node and its neighbour across the line, ref the
    line's unit direction) and, in 2D, curvature windows of four consecutive
    nodes.  Weights are drawn around ``weight``; some tuples reach the block
    boundary, whose fixed or constrained nodes stay frozen partners."""
    rng = np.random.default_rng(seed)
    ids = np.asarray(g.blocks[block])
    d = g.d
    sh = ids.shape

    def line(length: int):
        ax = int(rng.integers(d))
        start = [int(rng.integers(0, sh[k] - (length - 1 if k == ax else 0))) for k in range(d)]
        nodes = []
        for m in range(length):
            q = list(start)
            q[ax] += m
            nodes.append(int(ids[tuple(q)]))
        return ax, start, nodes

    def unit(v):
        return v / np.linalg.norm(v)

    nodes, kind, ref, axis, w = [], [], [], [], []
    for t in range(n_dir):
        k = t % 3
        if k == 1:  # line: a, c, b
            _ax, _st, nd = line(3)
            r = np.zeros(d)
        else:
            ax, st, nd = line(2)
            u = unit(g.X[nd[1]] - g.X[nd[0]])
            if k == 0:  # parallel: the segment's normal, tilted
                nrm = np.array([-u[1], u[0]]) if d == 2 else unit(np.cross(u, rng.normal(size=3)))
                r = unit(nrm + 0.3 * rng.normal(size=d))
            else:  # stem: n across the line at c, ref the line's direction
                other = (ax + 1 + int(rng.integers(d - 1))) % d
                c = list(st)
                c[other] = min(max(c[other], 1), sh[other] - 2)
                n = list(c)
                n[other] += 1 if rng.random() < 0.5 else -1
                nd = [int(ids[tuple(n)]), int(ids[tuple(c)])]
                r = unit(u + 0.2 * rng.normal(size=d))
        nodes.append(nd + [-1] * (4 - len(nd)))
        kind.append(k)
        ref.append(r)
        axis.append(np.zeros(d))
        w.append(weight * rng.uniform(0.5, 1.5))
    soft = {"directional": {"nodes": np.array(nodes, dtype=np.int32), "kind": np.array(kind, dtype=np.int32),
                            "ref": np.array(ref), "axis": np.array(axis), "weight": np.array(w), "eps": 1e-12}}
    if d == 2 and n_curv:
        cn, cw = [], []
        for _ in range(n_curv):
            cn.append(line(4)[2])
            cw.append(weight * rng.uniform(0.5, 1.5))
        soft["curvature"] = {"nodes": np.array(cn, dtype=np.int64), "weight": np.array(cw)}
    g.soft = soft
    g.name = g.name + "+soft"
    return g
