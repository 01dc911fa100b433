"""Builders for the sweep-context wire and the structured block tables.

The egg core consumes two dicts (``ctx_arrays`` and ``structured``) whose
format is fixed by the reference's pybind boundary:

* ``ctx_arrays = {"groups": [group], "energy_stencil": stencil}`` as assembled by
  ``egg/smoothing/flat_context.py:136-346`` (``build_flat_context``) and unpacked
  by ``src/bindings.cpp:332-489`` (``unpack_context``);
* ``structured = {interior_shapes, block_global_dof, halo_src_block,
  halo_src_padded, halo_dst_block, halo_dst_padded, sing_block,
  sing_logical}`` as packed by ``egg/smoothing/cpp_backend.py:679-691``.

This module produces the same dicts from per-block global-node-id arrays with
vectorised numpy, so tests and benchmarks can build inputs without the egg
Python package.  Conventions (kept identical because the wire is an interface):

* A block is an integer array of global node ids with shape ``(n_0, ..., n_{d-1})``;
  cells are enumerated block by block in C order.
* Corner index ``b`` in ``0 .. 2**d - 1`` packs per-axis offset bits with axis 0
  most significant; sample id ``= 2**d * cell + b``
  (``egg/smoothing/flat_context.py:40-121``).
* Sample ``(cell, b)`` has corner ``C[cell, b]``, axis-``k`` neighbour
  ``C[cell, b ^ bit_k]`` and sign ``+1`` if bit ``k`` of ``b`` is clear else ``-1``.
* A node at local corner ``a`` meets sample ``b`` of the same cell with role
  ``0`` (``a == b``), ``1 + k`` (``a ^ b == bit_k``) or ``-1`` otherwise.
* Interior-eligible DOFs (logical index in ``[1, n-2]`` on every axis of their
  block, target a uniform multiple of the identity) carry no stored samples:
  ``interior_block``/``interior_logical`` name them and ``P_of`` is 0
  (``egg/smoothing/flat_context.py:211-238``).
* Soft terms ride as per-DOF fixed-K tables on the group (``curv_*``,
  ``dir_*``) and as one whole-sample directional table on the energy stencil
  (``egg/smoothing/flat_context.py:293-345``); node ids stay global.

Extension (accepted by this repository's core only): ``compact=True`` emits the
energy stencil as ``{"num_samples": ns, "structured": 1, "W_inv": row}`` with no
per-sample index arrays, for the canonical cell stencil of the blocks.  The
reference core requires the explicit arrays (``compact=False``).
"""

from __future__ import annotations

import numpy as np

__all__ = [
    "build_flat_context",
    "axis_bits",
    "role_table",
    "cell_corner_ids",
    "cell_stencil",
    "flat_wire",
    "structured_tables",
    "free_mask_from_fixed",
]


def axis_bits(d: int) -> np.ndarray:
    """Corner-index bit of each axis (axis 0 is the most significant bit)."""
    return np.array([1 << (d - 1 - k) for k in range(d)], dtype=np.int64)


def role_table(d: int) -> np.ndarray:
    """``role[a, b]`` of local corner ``a`` in the sample at local corner ``b``."""
    nc = 1 << d
    bits = axis_bits(d)
    role = np.full((nc, nc), -1, dtype=np.int32)
    b = np.arange(nc)
    role[b, b] = 0
    for k in range(d):
        role[b, b ^ bits[k]] = 1 + k
    return role


def cell_corner_ids(blocks: list[np.ndarray], d: int) -> np.ndarray:
    """``C[cell, a]``: global id of local corner ``a`` of every cell, all blocks."""
    nc = 1 << d
    cols_all = []
    for ids in blocks:
        ids = np.asarray(ids)
        shp = ids.shape
        if any(s < 2 for s in shp):
            continue
        cols = []
        for a in range(nc):
            sl = tuple(
                slice((a >> (d - 1 - ax)) & 1, ((a >> (d - 1 - ax)) & 1) + shp[ax] - 1)
                for ax in range(d)
            )
            cols.append(ids[sl].reshape(-1))
        cols_all.append(np.stack(cols, axis=1))
    if not cols_all:
        return np.zeros((0, nc), dtype=np.int64)
    return np.concatenate(cols_all).astype(np.int64)


def cell_stencil(blocks: list[np.ndarray], d: int):
    """Per-sample ``(gc, gn[d], s[d])`` in canonical sample order."""
    nc = 1 << d
    bits = axis_bits(d)
    C = cell_corner_ids(blocks, d)
    b = np.arange(nc)
    sgn = np.where((b[:, None] & bits[None, :]) == 0, 1.0, -1.0)  # (nc, d)
    gc = C.reshape(-1)
    gn = [C[:, b ^ bits[k]].reshape(-1) for k in range(d)]
    s = [np.tile(sgn[:, k], C.shape[0]) for k in range(d)]
    return C, gc, gn, s


def free_mask_from_fixed(n_nodes: int, fixed_ids) -> np.ndarray:
    m = np.ones(n_nodes, dtype=bool)
    m[np.asarray(fixed_ids, dtype=np.int64)] = False
    return m


# Entity partitions of constrained DOFs: tag -> (partition name, kFields),
# the reference's frozen tags and packed record widths (src/entity_soa.hpp:37-56,
# src/geometry.hpp:1760-1928).
ENTITY_KINDS = {1: ("line_seg", 4), 2: ("circle", 3), 3: ("ellipse", 4), 5: ("plane", 9), 6: ("circle_arc", 6),
                7: ("ellipse_arc", 8), 8: ("quad_bezier", 8), 9: ("cubic_bezier", 10), 15: ("line_rail", 4),
                16: ("line_rail3", 6), 4: ("sphere", 10), 12: ("cylinder", 10), 13: ("line3", 8),
                10: ("bspline", 6), 11: ("composite", 2), 14: ("bsplinesurf", 9)}


def flat_wire(
    blocks: list[np.ndarray],
    free_mask: np.ndarray,
    d: int,
    *,
    w_inv: np.ndarray | None = None,
    compact: bool = False,
    constraints: dict | None = None,
    directional: dict | None = None,
    curvature: dict | None = None,
    device: str | None = None,
) -> dict:
    """The ``{"groups", "energy_stencil"}`` wire for Free DOFs and, optionally,
    constrained boundary DOFs.

    ``w_inv`` is one ``(d, d)`` inverse target shared by every sample (default
    identity) or ``(ns, d, d)`` per sample in canonical order.  Mirrors
    ``build_flat_context`` (``egg/smoothing/flat_context.py:136-346``) without
    interface samples.  ``constraints`` maps a global
    node id (not Free) to ``(tag, record)`` or ``(tag, record, seg)``, seg the
    entity's variable-length fields (a B-spline's knots, control points and
    weights), sent as one ``{data, off}`` CSR field each: the node becomes a moving DOF on
    that entity (``ENTITY_KINDS``), with a stored patch, in one SoA partition
    per tag whose packed records follow the partition's ``dof_local`` order.
    ``compact`` drops the energy-stencil index arrays (see module docstring) and
    sends a uniform target as one shared row.
    ``directional`` (``nodes`` (n, 4) -1 padded, ``kind``, ``ref`` (n, d),
    ``axis`` (n, d), ``weight``, ``eps``) and ``curvature`` (``nodes`` (W, 4),
    ``weight``) add the soft-term tables (``soft_tables``).
    ``device`` (``"auto"``, ``"gpu"`` or ``"cuda:N"``) builds the index arrays
    -- interior classification, the stored DOFs' membership rows sorted by
    node, ``P_of`` and the energy stencil -- with the core's kernels
    (``cpp_core.wire_build``); the result is identical to the host build's.
    """
    constraints = constraints or {}
    con_ids = np.array(sorted(constraints), dtype=np.int64)
    if con_ids.size and np.asarray(free_mask)[con_ids].any():
        raise ValueError("flat_wire: a constrained node is also marked Free")
    blocks = [np.asarray(b) for b in blocks]
    nc = 1 << d
    dd = d * d
    N = int(free_mask.shape[0])
    if w_inv is None:
        w_inv = np.eye(d)
    w_inv = np.asarray(w_inv, dtype=np.float64)
    uniform_w = w_inv.shape == (d, d)
    w0 = w_inv if uniform_w else (w_inv[0] if len(w_inv) else np.eye(d))
    synth_interior = bool(
        np.allclose(w0, w0[0, 0] * np.eye(d)) and (uniform_w or np.allclose(w_inv, w0))
    )

    moving = np.asarray(free_mask, dtype=bool).copy()
    moving[con_ids] = True
    stored = None
    if con_ids.size:
        stored = np.zeros(N, dtype=bool)
        stored[con_ids] = True
    if device is None:
        arr = _host_arrays(blocks, moving, stored, d, synth_interior, not compact)
    else:
        arr = _device_arrays(blocks, moving, stored, d, synth_interior, not compact, device)
    ns = int(arr["num_samples"])

    def fields(pre: str, sid, rows: int, *, uniform_out: bool) -> dict:
        out = {"gc": arr[pre + "gc"]}
        for k in range(d):
            out[f"gn{k}"] = arr[f"{pre}gn{k}"]
            out[f"s{k}"] = arr[f"{pre}s{k}"]
        if uniform_w and uniform_out:
            W = w_inv.reshape(1, dd)
        elif uniform_w:
            W = np.broadcast_to(w_inv, (rows, d, d)).reshape(-1, dd)
        else:
            W = w_inv[sid].reshape(-1, dd)
        out["W_inv"] = np.ascontiguousarray(W, dtype=np.float64)
        return out

    groups = []
    dofs = arr["dof_idx"]
    if dofs.size:
        g = {
            "D": int(dofs.size),
            "role": arr["role"],
            "dof_idx": dofs,
            "P_of": arr["P_of"],
            "interior_block": arr["interior_block"],
            "interior_logical": arr["interior_logical"],
            "entities": {
                "free": {
                    "tag": 0,
                    "kFields": 0,
                    "dof_local": np.flatnonzero(np.asarray(free_mask)[dofs]).astype(np.int32),
                    "records": np.zeros(0, dtype=np.float64),
                }
            },
        }
        for tag in sorted({int(constraints[int(n)][0]) for n in con_ids}):
            name, kf = ENTITY_KINDS[tag]
            nodes = [int(n) for n in con_ids if int(constraints[int(n)][0]) == tag]
            local = np.searchsorted(dofs, np.array(nodes, dtype=np.int64)).astype(np.int32)
            rec = np.array([np.asarray(constraints[n][1], dtype=np.float64)[:kf] for n in nodes])
            g["entities"][name] = {"tag": tag, "kFields": kf, "dof_local": local,
                                   "records": np.ascontiguousarray(rec.reshape(-1))}
            if len(constraints[nodes[0]]) > 2:  # segmented fields: (knots, ctrl, weights) per node
                seg = []
                for k in range(len(constraints[nodes[0]][2])):
                    parts = [np.asarray(constraints[n][2][k], dtype=np.float64).ravel() for n in nodes]
                    off = np.concatenate([[0], np.cumsum([len(x) for x in parts])]).astype(np.int32)
                    seg.append({"data": np.concatenate(parts) if parts else np.zeros(0), "off": off})
                g["entities"][name]["seg"] = seg

        g.update(fields("", arr["sid"], int(arr["role"].size), uniform_out=True))
        g.update(soft_tables(moving, d, directional=directional, curvature=curvature))
        groups.append(g)

    if compact:
        if not uniform_w:
            raise ValueError("compact wire requires a uniform target")
        es = {"num_samples": int(ns), "structured": 1, "W_inv": w_inv.reshape(1, dd).copy()}
    else:
        es = {"num_samples": ns}
        es.update(fields("es_", np.arange(ns, dtype=np.int64), ns, uniform_out=True))
    if directional is not None and len(directional["kind"]):
        es.update({
            "dir_num": int(len(directional["kind"])),
            "dir_eps": float(directional["eps"]),
            "dir_nodes": np.ascontiguousarray(np.asarray(directional["nodes"], dtype=np.int32)),
            "dir_kind": np.ascontiguousarray(np.asarray(directional["kind"], dtype=np.int32)),
            "dir_ref": np.ascontiguousarray(np.asarray(directional["ref"], dtype=np.float64)),
            "dir_axis": np.ascontiguousarray(np.asarray(directional["axis"], dtype=np.float64)),
            "dir_weight": np.ascontiguousarray(np.asarray(directional["weight"], dtype=np.float64)),
        })
    return {"groups": groups, "energy_stencil": es}


def _host_arrays(blocks, moving, stored, d: int, synth_interior: bool, energy_arrays: bool) -> dict:
    """Index arrays of the wire, vectorised numpy (the layout of
    ``egg/smoothing/flat_context.py:211-272``): interior-eligible nodes name
    (block, logical); the membership rows (cell, a, b) of moving, non-interior
    nodes, stably sorted by node; the energy stencil in sample order."""
    N = moving.shape[0]
    nc = 1 << d
    node_block = np.full(N, -1, dtype=np.int32)
    node_logical = np.zeros((N, d), dtype=np.int32)
    if synth_interior:
        for bi, ids in enumerate(blocks):
            sh = ids.shape
            if any(s < 3 for s in sh):
                continue
            inner = ids[tuple(slice(1, s - 1) for s in sh)].reshape(-1)
            grids = np.meshgrid(*[np.arange(1, s - 1, dtype=np.int32) for s in sh], indexing="ij")
            node_block[inner] = bi
            node_logical[inner] = np.stack([g.reshape(-1) for g in grids], axis=1)
    if stored is not None:
        node_block[stored] = -1  # constrained nodes always take a stored patch
    node_interior = node_block >= 0

    C = cell_corner_ids(blocks, d)
    ns = C.shape[0] * nc
    bits = axis_bits(d)
    bidx = np.arange(nc)
    sgn = np.where((bidx[:, None] & bits[None, :]) == 0, 1.0, -1.0)
    role = role_table(d)

    # Membership only for stored-patch DOFs (moving, not interior-eligible):
    # restrict to cells that touch such a node, so large grids with few stored
    # DOFs never materialise the full node x sample table.
    stored_node = moving & ~node_interior
    touch = stored_node[C]  # (ncell, nc)
    cells = np.flatnonzero(touch.any(axis=1))
    Ct = C[cells]  # (m, nc)
    # Rows (cell, a, b) restricted to stored nodes at corner a.
    m_node = np.repeat(Ct[:, :, None], nc, axis=2).reshape(-1)
    m_sid = (nc * cells[:, None, None] + bidx[None, None, :]).repeat(nc, axis=1).reshape(-1)
    m_role = np.tile(role.reshape(-1), cells.shape[0])
    keep = stored_node[m_node]
    m_node, m_sid, m_role = m_node[keep], m_sid[keep], m_role[keep]
    perm = np.argsort(m_node, kind="stable")
    m_node, m_sid, m_role = m_node[perm], m_sid[perm], m_role[perm]

    dofs = np.flatnonzero(moving)
    P_of = np.zeros(dofs.size, dtype=np.int32)
    if m_node.size:
        uniq, cnt = np.unique(m_node, return_counts=True)
        P_of[np.searchsorted(dofs, uniq)] = cnt
    out = {
        "num_samples": ns,
        "dof_idx": dofs.astype(np.int32),
        "P_of": P_of,
        "interior_block": np.ascontiguousarray(node_block[dofs]),
        "interior_logical": np.ascontiguousarray(node_logical[dofs]),
        "role": m_role.astype(np.int32),
        "sid": m_sid,
    }

    def rows(pre: str, sid: np.ndarray) -> None:
        cell = sid // nc
        b = sid % nc
        out[pre + "gc"] = C[cell, b].astype(np.int32)
        for k in range(d):
            out[f"{pre}gn{k}"] = C[cell, b ^ bits[k]].astype(np.int32)
            out[f"{pre}s{k}"] = sgn[b, k].astype(np.float64)

    rows("", m_sid)
    if energy_arrays:
        rows("es_", np.arange(ns, dtype=np.int64))
    return out


def _device_arrays(blocks, moving, stored, d: int, synth_interior: bool, energy_arrays: bool, device: str) -> dict:
    """The same index arrays built on the GPU (``cpp_core.wire_build``)."""
    from . import load_core

    core = load_core()
    shapes = np.array([b.shape for b in blocks], dtype=np.int32).reshape(-1)
    ids = (np.concatenate([np.asarray(b, dtype=np.int64).reshape(-1) for b in blocks])
           if blocks else np.zeros(0, dtype=np.int64))
    return core.wire_build(d, shapes, ids, moving.view(np.uint8),
                           None if stored is None else stored.view(np.uint8),
                           synth_interior=synth_interior, energy_arrays=energy_arrays, device=device)


def build_flat_context(blocks, free_mask, dof_entities, d: int, *, w_inv, interface=None, curvature=None,
                       directional=None, device: str = "auto") -> dict:
    """Drop-in for the reference's ``egg.smoothing.flat_context.build_flat_context``
    (``flat_context.py:136-346``; same arguments and result) whose index
    arrays -- interior classification, the moving DOFs' membership rows
    sorted by node, ``P_of`` and the energy stencil -- are built on the GPU
    (``cpp_core.wire_build``).  The entity partitions and the soft-term
    tables come from the reference's own packers
    (``egg.geometry.entity_soa.group_entities_by_type``,
    ``egg.smoothing.interface_c2.curvature_dof_table``,
    ``egg.smoothing.directional.directional_dof_table`` /
    ``directional_energy_table``), so the reference's ``egg`` package must
    be importable.  ``free_mask`` marks every moving DOF, ``dof_entities``
    maps constrained ones to their entity, as in the reference.  Interface
    samples (the composed orthogonality term) are not built here and raise
    ``NotImplementedError``; pass them to the reference builder."""
    if interface is not None and len(interface) > 0:
        raise NotImplementedError("build_flat_context (device): interface samples are not supported")
    from egg.geometry.entity_soa import group_entities_by_type

    blocks = [np.asarray(b) for b in blocks]
    moving = np.asarray(free_mask, dtype=bool)
    dd = d * d
    w_inv = np.asarray(w_inv, dtype=np.float64)
    uniform_w = w_inv.shape == (d, d)
    w0 = w_inv if uniform_w else (w_inv[0] if len(w_inv) else np.eye(d))
    synth_interior = bool(np.allclose(w0, w0[0, 0] * np.eye(d)) and (uniform_w or np.allclose(w_inv, w0)))
    arr = _device_arrays(blocks, moving, None, d, synth_interior, True, device)
    ns = int(arr["num_samples"])

    def fields(pre: str, sid) -> dict:
        out = {"gc": arr[pre + "gc"]}
        for k in range(d):
            out[f"gn{k}"] = arr[f"{pre}gn{k}"]
            out[f"s{k}"] = arr[f"{pre}s{k}"]
        out["W_inv"] = np.ascontiguousarray(w_inv.reshape(1, dd) if uniform_w else w_inv[sid].reshape(-1, dd))
        return out

    groups = []
    dofs = arr["dof_idx"]
    if dofs.size:
        g = {
            "D": int(dofs.size),
            "role": arr["role"],
            "dof_idx": dofs,
            "P_of": arr["P_of"],
            "interior_block": arr["interior_block"],
            "interior_logical": arr["interior_logical"],
            "entities": group_entities_by_type(dofs.astype(np.int64).tolist(), dof_entities, d=d),
        }
        g.update(fields("", arr["sid"]))
        if curvature is not None and len(curvature) > 0:
            from egg.smoothing.interface_c2 import curvature_dof_table

            tab = curvature_dof_table(moving, curvature)
            if tab:
                g["curv_k"] = tab["curv_k"]
                for key in ("curv_nodes", "curv_slot", "curv_weight"):
                    g[key] = np.ascontiguousarray(tab[key].reshape(-1))
        if directional is not None and directional.n > 0:
            from egg.smoothing.directional import directional_dof_table

            tab = directional_dof_table(moving, directional)
            if tab:
                g["dir_k"] = tab["dir_k"]
                g["dir_eps"] = tab["dir_eps"]
                for key in ("dir_nodes", "dir_slot", "dir_kind", "dir_ref", "dir_axis", "dir_weight"):
                    g[key] = np.ascontiguousarray(tab[key].reshape(-1))
        groups.append(g)
    es = {"num_samples": ns}
    es.update(fields("es_", np.arange(ns, dtype=np.int64)))
    if directional is not None and directional.n > 0:
        from egg.smoothing.directional import directional_energy_table

        tab = directional_energy_table(directional)
        if tab:
            es["dir_num"] = tab["dir_num"]
            es["dir_eps"] = tab["dir_eps"]
            for key in ("dir_nodes", "dir_axis", "dir_ref"):
                es[key] = np.ascontiguousarray(tab[key].reshape(-1))
            es["dir_kind"] = tab["dir_kind"]
            es["dir_weight"] = tab["dir_weight"]
    return {"groups": groups, "energy_stencil": es}


DIR_ARITY = {0: 2, 1: 3, 2: 2}  # parallel, line, stem; other kinds are reserved (arity 0)


def soft_tables(moving: np.ndarray, d: int, *, directional: dict | None = None,
                curvature: dict | None = None) -> dict:
    """Per-DOF fixed-K soft-term tables of the group (wire layout of
    ``egg/smoothing/directional.py:381-437`` and
    ``egg/smoothing/interface_c2.py:233-279``).

    For each moving DOF in ascending order, every term it takes part in is
    listed with the DOF's slot in the term, in term order, padded to the
    widest DOF's count K with slot -1.  Node ids stay global.  Returns
    ``curv_k``/``curv_nodes`` (ndof, K, 4)/``curv_slot``/``curv_weight`` and
    ``dir_k``/``dir_eps``/``dir_nodes`` (ndof, K, 4)/``dir_slot``/``dir_kind``/
    ``dir_ref`` and ``dir_axis`` (ndof, K, d)/``dir_weight``; nothing for an
    absent or empty term set.
    """
    if (directional is None or not len(directional["kind"])) and (curvature is None or not len(curvature["weight"])):
        return {}
    moving = np.asarray(moving, dtype=bool)
    dofs = np.flatnonzero(moving)
    pos = np.full(moving.shape[0], -1, dtype=np.int64)
    pos[dofs] = np.arange(dofs.size)
    out: dict = {}

    def listing(nodes: np.ndarray, arity) -> list:
        per = [[] for _ in range(dofs.size)]
        for t in range(nodes.shape[0]):
            for slot in range(arity(t)):
                nd = int(nodes[t, slot])
                if nd >= 0 and moving[nd]:
                    per[int(pos[nd])].append((t, slot))
        return per

    if curvature is not None and len(curvature["weight"]) and dofs.size:
        cn = np.asarray(curvature["nodes"], dtype=np.int64).reshape(-1, 4)
        cw = np.asarray(curvature["weight"], dtype=np.float64)
        per = listing(cn, lambda t: 4)
        K = max(len(e) for e in per)
        if K:
            nodes = np.full((dofs.size, K, 4), -1, dtype=np.int32)
            slot = np.full((dofs.size, K), -1, dtype=np.int32)
            w = np.zeros((dofs.size, K))
            for i, e in enumerate(per):
                for j, (t, sl) in enumerate(e):
                    nodes[i, j], slot[i, j], w[i, j] = cn[t], sl, cw[t]
            out.update({"curv_k": int(K), "curv_nodes": nodes.reshape(-1), "curv_slot": slot.reshape(-1),
                        "curv_weight": w.reshape(-1)})
    if directional is not None and len(directional["kind"]) and dofs.size:
        dn = np.asarray(directional["nodes"], dtype=np.int64).reshape(-1, 4)
        dk = np.asarray(directional["kind"], dtype=np.int64)
        dr = np.asarray(directional["ref"], dtype=np.float64).reshape(-1, d)
        da = np.asarray(directional["axis"], dtype=np.float64).reshape(-1, d)
        dw = np.asarray(directional["weight"], dtype=np.float64)
        per = listing(dn, lambda t: DIR_ARITY.get(int(dk[t]), 0))
        K = max(len(e) for e in per)
        if K:
            nodes = np.full((dofs.size, K, 4), -1, dtype=np.int32)
            slot = np.full((dofs.size, K), -1, dtype=np.int32)
            kind = np.zeros((dofs.size, K), dtype=np.int32)
            ref = np.zeros((dofs.size, K, d))
            axis = np.zeros((dofs.size, K, d))
            w = np.zeros((dofs.size, K))
            for i, e in enumerate(per):
                for j, (t, sl) in enumerate(e):
                    nodes[i, j], slot[i, j], kind[i, j] = dn[t], sl, dk[t]
                    ref[i, j], axis[i, j], w[i, j] = dr[t], da[t], dw[t]
            out.update({"dir_k": int(K), "dir_eps": float(directional["eps"]), "dir_nodes": nodes.reshape(-1),
                        "dir_slot": slot.reshape(-1), "dir_kind": kind.reshape(-1), "dir_ref": ref.reshape(-1),
                        "dir_axis": axis.reshape(-1), "dir_weight": w.reshape(-1)})
    return out


def structured_tables(blocks: list[np.ndarray]) -> dict:
    """The ``structured`` dict for hand-assembled blocks (shared-id twin matching).

    Follows ``build_structured_context_from_block_maps``
    (``egg/smoothing/cpp_backend.py:120-244``): a face node that also lives in
    another block gets a ghost entry filled by the node one step behind its twin
    (the lowest-block copy of that node when it is itself shared); ambiguous
    cases are left out.  Singularity tables stay empty.
    """
    blocks = [np.asarray(b) for b in blocks]
    d = blocks[0].ndim
    shapes = [tuple(int(s) for s in b.shape) for b in blocks]
    flat = [np.ascontiguousarray(b.reshape(-1), dtype=np.int32) for b in blocks]
    n_ids = max(int(f.max()) for f in flat if f.size) + 1
    counts = np.zeros(n_ids, dtype=np.int64)
    for f in flat:
        counts += np.bincount(f, minlength=n_ids)
    shared = counts > 1
    where: dict[int, list] = {}
    for bi, ids in enumerate(blocks):
        for logical in zip(*np.nonzero(shared[ids])):
            li = tuple(int(c) for c in logical)
            where.setdefault(int(ids[li]), []).append((bi, li))
    member = []
    for f in flat:
        m = np.zeros(n_ids, dtype=bool)
        m[f] = True
        member.append(m)

    def behind(dst_block: int, gid: int):
        found = None
        loc = None
        for bj, lj in where.get(gid, ()):
            if bj == dst_block:
                continue
            shp = shapes[bj]
            for ax in range(d):
                if lj[ax] == 0:
                    step = 1
                elif lj[ax] == shp[ax] - 1:
                    step = -1
                else:
                    continue
                inner = list(lj)
                inner[ax] += step
                g_in = int(blocks[bj][tuple(inner)])
                if member[dst_block][g_in]:
                    continue
                if found is not None and found != g_in:
                    return None
                found = g_in
                loc = (bj, tuple(inner))
        if found is None:
            return None
        if shared[found]:
            return min(where[found])
        return loc

    sb, sp, db, dp = [], [], [], []
    for bi, ids in enumerate(blocks):
        shp = shapes[bi]
        for ax in range(d):
            for side in (0, 1):
                fixed = 0 if side == 0 else shp[ax] - 1
                face = np.take(ids, fixed, axis=ax)
                for free_idx in zip(*np.nonzero(shared[face])):
                    gid = int(face[free_idx])
                    logical = list(free_idx[:ax]) + [fixed] + list(free_idx[ax:])
                    hit = behind(bi, gid)
                    if hit is None:
                        continue
                    bj, inner = hit
                    ghost = [c + 1 for c in logical]
                    ghost[ax] = 0 if side == 0 else shp[ax] + 1
                    sb.append(bj)
                    sp.append(tuple(c + 1 for c in inner))
                    db.append(bi)
                    dp.append(tuple(ghost))
    rows = lambda v: np.asarray(v, dtype=np.int32).reshape(-1, d)  # noqa: E731
    return {
        "interior_shapes": [np.asarray(s, dtype=np.int32) for s in shapes],
        "block_global_dof": flat,
        "halo_src_block": np.asarray(sb, dtype=np.int32),
        "halo_src_padded": rows(sp),
        "halo_dst_block": np.asarray(db, dtype=np.int32),
        "halo_dst_padded": rows(dp),
        "sing_block": np.zeros(0, dtype=np.int32),
        "sing_logical": np.zeros((0, d), dtype=np.int32),
    }
