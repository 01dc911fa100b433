"""Control-net wire of one block for the reduced Gauss-Newton smoother.

The block's nodes become X = M C + b:

- M is the tensor product of per-axis clamped B-spline bases (uniform
  interior knots, node parameters uniform in [0, 1]). The basis values are
  the standard triangular recurrence of the nonzero B-splines on a knot
  span (Piegl & Tiller, *The NURBS Book*, algorithms A2.1/A2.2).
- C is fitted to the block's nodes facet by facet: corners exactly, then
  every facet's interior controls by least squares with the already-set
  lower-dimensional controls frozen. Per-axis pseudo-inverses are applied
  as mode products (the slab's free controls are a tensor product of
  per-axis interior ranges).
- b is the Boolean-sum offset: the boundary mismatch X0 - M C, extended
  inward by transfinite interpolation (sum of the per-axis linear blends
  minus (D - 1) times the multilinear corner blend). Boundary nodes are
  then exact and b depends only on the frozen boundary controls.

The wire dict has the keys of egg/smoothing/control_backend.py:76
build_control_wire (block, ctrl_shape, k_supp, C0, free_idx, b, off{k},
wt{k}): each axis ships a band of k_supp weights per node and the
offset of its first control.
"""

from __future__ import annotations

from itertools import product

import numpy as np


def clamped_knots(n_ctrl: int, degree: int) -> np.ndarray:
    """degree + 1 repeated knots at 0 and 1, evenly spaced interior knots."""
    if n_ctrl < degree + 1:
        raise ValueError(f"need n_ctrl >= degree + 1, got {n_ctrl} controls for degree {degree}")
    m = n_ctrl - degree - 1
    inner = np.arange(1, m + 1, dtype=float) / (m + 1)
    return np.concatenate([np.zeros(degree + 1), inner, np.ones(degree + 1)])


def _span(n: int, p: int, u: float, U: np.ndarray) -> int:
    # knot span holding u, clamped to [p, n] so that u = 0 and u = 1 are exact
    if u >= U[n + 1]:
        return n
    if u <= U[p]:
        return p
    lo, hi = p, n + 1
    while hi - lo > 1:
        mid = (lo + hi) // 2
        if u < U[mid]:
            hi = mid
        else:
            lo = mid
    return lo


def _nonzero_basis(i: int, u: float, p: int, U: np.ndarray) -> np.ndarray:
    # the p + 1 B-splines N_{i-p..i} nonzero on span i, by the triangular recurrence
    N = np.zeros(p + 1)
    left = np.zeros(p + 1)
    right = np.zeros(p + 1)
    N[0] = 1.0
    for j in range(1, p + 1):
        left[j] = u - U[i + 1 - j]
        right[j] = U[i + j] - u
        carry = 0.0
        for r in range(j):
            tmp = N[r] / (right[r + 1] + left[j - r])
            N[r] = carry + right[r + 1] * tmp
            carry = left[j - r] * tmp
        N[j] = carry
    return N


def basis_matrix(n_ctrl: int, degree: int, params) -> np.ndarray:
    """(len(params), n_ctrl) value matrix of the clamped basis (rows sum to 1)."""
    U = clamped_knots(n_ctrl, degree)
    params = np.asarray(params, dtype=float)
    B = np.zeros((params.size, n_ctrl))
    for k, u in enumerate(params):
        i = _span(n_ctrl - 1, degree, float(u), U)
        B[k, i - degree : i + 1] = _nonzero_basis(i, float(u), degree, U)
    return B


def axis_bases(node_shape, ctrl_shape, degree: int = 3) -> list[np.ndarray]:
    return [basis_matrix(int(c), degree, np.linspace(0.0, 1.0, int(n))) for n, c in zip(node_shape, ctrl_shape)]


def _mode(mats, T: np.ndarray) -> np.ndarray:
    for k, A in enumerate(mats):
        T = np.moveaxis(np.tensordot(A, T, axes=([1], [k])), 0, k)
    return T


def prolong(bases, C: np.ndarray) -> np.ndarray:
    """M C: control lattice (ctrl_shape + (d,)) -> nodes (node_shape + (d,))."""
    return _mode(bases, np.asarray(C, dtype=float))


def _slab(offset, shape):
    return tuple(0 if o == -1 else (n - 1 if o == 1 else slice(None)) for o, n in zip(offset, shape))


def fit_lattice(bases, X0: np.ndarray) -> np.ndarray:
    """Facet-by-facet least-squares control lattice for the nodes X0."""
    d = len(bases)
    ctrl_shape = tuple(B.shape[1] for B in bases)
    node_shape = tuple(B.shape[0] for B in bases)
    C = np.zeros(ctrl_shape + (d,))
    pinv = {}
    offsets = [o for o in product((-1, 0, 1), repeat=d) if any(o)]
    offsets.sort(key=lambda o: sum(1 for v in o if v == 0))  # corners, edges, faces
    for off in offsets + [(0,) * d]:
        span = [k for k in range(d) if off[k] == 0]
        cs, ns = _slab(off, ctrl_shape), _slab(off, node_shape)
        if not span:
            C[cs] = X0[ns]
            continue
        slab = np.array(C[cs])
        inner = tuple(slice(1, -1) for _ in span)
        slab[inner] = 0.0
        rhs = X0[ns] - _mode([bases[k] for k in span], slab)
        for k in span:
            if k not in pinv:
                pinv[k] = np.linalg.pinv(bases[k][:, 1:-1])
        slab[inner] = _mode([pinv[k] for k in span], rhs)
        C[cs] = slab
    return C


def boundary_mask(shape) -> np.ndarray:
    """Lattice points on the boundary of a box of the given shape."""
    m = np.zeros(tuple(shape), dtype=bool)
    for k in range(len(shape)):
        sl = [slice(None)] * len(shape)
        sl[k] = 0
        m[tuple(sl)] = True
        sl[k] = shape[k] - 1
        m[tuple(sl)] = True
    return m


def _blend(F: np.ndarray) -> np.ndarray:
    # sum of per-axis linear blends minus (D - 1) times the multilinear corner blend
    d = F.ndim - 1
    t = [np.linspace(0.0, 1.0, n) for n in F.shape[:-1]]

    def lerp(G, ax):
        sh = [1] * (d + 1)
        sh[ax] = F.shape[ax]
        s = t[ax].reshape(sh)
        return (1.0 - s) * np.take(G, [0], axis=ax) + s * np.take(G, [-1], axis=ax)

    total = lerp(F, 0)
    for ax in range(1, d):
        total = total + lerp(F, ax)
    corner = F
    for ax in range(d):
        corner = lerp(corner, ax)
    return total - (d - 1) * corner


def boolean_sum_offset(bases, C: np.ndarray, X0: np.ndarray) -> np.ndarray:
    """b: boundary mismatch X0 - M C, extended inward by transfinite blending."""
    node_shape = tuple(B.shape[0] for B in bases)
    bm = boundary_mask(node_shape)
    delta = np.zeros(node_shape + (len(bases),))
    delta[bm] = (X0 - prolong(bases, C))[bm]
    b = np.array(delta)
    inner = tuple(slice(1, -1) for _ in node_shape)
    b[inner] = _blend(delta)[inner]
    return b


def _band(B: np.ndarray, k_supp: int):
    n_node, n_ctrl = B.shape
    if n_ctrl < k_supp:
        raise ValueError(f"axis has {n_ctrl} controls < support width {k_supp}")
    off = np.empty(n_node, dtype=np.int32)
    wt = np.zeros((n_node, k_supp))
    for i in range(n_node):
        nz = np.flatnonzero(B[i] != 0.0)
        first = min(int(nz[0]) if nz.size else 0, n_ctrl - k_supp)
        if nz.size and int(nz[-1]) - first + 1 > k_supp:
            raise ValueError(f"basis row {i} is wider than k_supp {k_supp}")
        off[i] = first
        wt[i] = B[i, first : first + k_supp]
    return off, wt.reshape(-1)


def control_wire(block_nodes: np.ndarray, ctrl_shape, *, degree: int = 3, block: int = 0) -> dict:
    """Wire dict of a net fitted to one block's nodes (node_shape + (d,)).

    Boundary controls are fixed, every other control is free."""
    X0 = np.asarray(block_nodes, dtype=float)
    d = X0.shape[-1]
    node_shape = X0.shape[:-1]
    ctrl_shape = tuple(int(c) for c in ctrl_shape)
    bases = axis_bases(node_shape, ctrl_shape, degree)
    C0 = fit_lattice(bases, X0)
    b = boolean_sum_offset(bases, C0, X0)
    free = ~boundary_mask(ctrl_shape)
    k_supp = degree + 1
    wire = {
        "block": int(block),
        "ctrl_shape": np.asarray(ctrl_shape, dtype=np.int32),
        "k_supp": int(k_supp),
        "C0": np.ascontiguousarray(C0).reshape(-1),
        "free_idx": np.flatnonzero(free.reshape(-1)).astype(np.int32),
        "b": np.ascontiguousarray(b).reshape(-1),
    }
    for k in range(d):
        wire[f"off{k}"], wire[f"wt{k}"] = _band(bases[k], k_supp)
    return wire


def grid_block_nodes(grid, block: int) -> np.ndarray:
    """A block's node positions (node_shape + (d,)) from a configs.Grid."""
    ids = grid.blocks[block]
    return grid.X[ids.reshape(-1)].reshape(ids.shape + (grid.d,))
