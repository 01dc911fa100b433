"""Python side of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and bench.py's ``cpu_baseline`` /
``--impl reference`` legs use this module, and only as the checker or the
timed CPU baseline; the egg_b200 product never imports it.

* :func:`load` builds (gcc) and loads ``egg_oracle.c`` -> ``oracle/_build/``;
* :func:`patches_for` expands a grid into explicit per-DOF patches with the
  reference's semantics (``egg/smoothing/flat_context.py:136-346`` membership
  order; structured-interior DOFs see an identity target,
  ``src/structured_patch.hpp:175-185``);
* :func:`run` / :func:`energy` run the restated block-Jacobi sweep;
* :func:`load_ref` loads the reference core built from source by
  ``oracle/build_ref.sh`` (``oracle/_ref/{fp64,fp32}``) when present.
"""

from __future__ import annotations

import ctypes as C
import importlib.util
import os
import subprocess
import sysconfig
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
BUILD = HERE / "_build"
SRC = HERE / "egg_oracle.c"
LIB = BUILD / "liboracle.so"

_lib = None


def build(force: bool = False) -> Path:
    if force or not LIB.exists() or LIB.stat().st_mtime < SRC.stat().st_mtime:
        BUILD.mkdir(exist_ok=True)
        tmp = LIB.with_suffix(".tmp")
        subprocess.run(
            ["gcc", "-O2", "-ffp-contract=off", "-shared", "-fPIC", "-std=c11", str(SRC), "-o", str(tmp), "-lm"],
            check=True,
        )
        tmp.replace(LIB)
    return LIB


def load():
    global _lib
    if _lib is None:
        build()
        lib = C.CDLL(str(LIB))
        P = C.c_void_p
        I64 = C.c_int64
        lib.oracle_run2d.restype = I64
        lib.oracle_run2d.argtypes = [C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, I64, P, I64] + [P] * 10 + [
            I64] + [P] * 6 + [I64, P, P, P]
        lib.oracle_energy2d.restype = None
        lib.oracle_energy2d.argtypes = [C.c_int, C.c_double, P, I64] + [P] * 6 + [I64, P, P, P]
        lib.oracle_metric2d.restype = None
        lib.oracle_metric2d.argtypes = [C.c_int, C.c_double, P, P, P, P]
        lib.oracle_patch2d.restype = None
        lib.oracle_patch2d.argtypes = [C.c_int, C.c_double, P, C.c_int32] + [P] * 7 + [P] * 5
        lib.oracle_metric3d.restype = None
        lib.oracle_metric3d.argtypes = [C.c_int, C.c_double, P, P, P, P]
        lib.oracle_run3d.restype = I64
        lib.oracle_run3d.argtypes = [C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, I64, P, I64] + [P] * 11 + [
            I64] + [P] * 8 + [I64, P, P]
        lib.oracle_energy3d.restype = None
        lib.oracle_energy3d.argtypes = [C.c_int, C.c_double, P, I64] + [P] * 8 + [I64, P, P]
        _lib = lib
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


KIND = {"barrier": 0, "shape": 0, "untangle": 1, "shape_size": 2}


def metric(t, kind="shape", delta=0.0):
    lib = load()
    t = np.ascontiguousarray(t, dtype=np.float64)
    mu = np.zeros(1)
    g = np.zeros(4)
    H = np.zeros(16)
    lib.oracle_metric2d(KIND[kind], float(delta), _p(t), _p(mu), _p(g), _p(H))
    return float(mu[0]), g, H


def patch(X, gc, gn0, gn1, s0, s1, W, role, kind="shape", delta=0.0):
    lib = load()
    X = np.ascontiguousarray(X, dtype=np.float64).ravel()
    ints = [np.ascontiguousarray(a, dtype=np.int32) for a in (gc, gn0, gn1, role)]
    reals = [np.ascontiguousarray(a, dtype=np.float64).ravel() for a in (s0, s1, W)]
    g, h, e, md, st = np.zeros(2), np.zeros(4), np.zeros(1), np.zeros(1), np.zeros(2)
    lib.oracle_patch2d(KIND[kind], float(delta), _p(X), len(ints[0]), _p(ints[0]), _p(ints[1]), _p(ints[2]),
                       _p(reals[0]), _p(reals[1]), _p(reals[2]), _p(ints[3]), _p(g), _p(h), _p(e), _p(md), _p(st))
    return g, h, float(e[0]), float(md[0]), st


def metric3(t, kind="shape", delta=0.0):
    lib = load()
    t = np.ascontiguousarray(t, dtype=np.float64)
    mu, g, H = np.zeros(1), np.zeros(9), np.zeros(81)
    lib.oracle_metric3d(KIND[kind], float(delta), _p(t), _p(mu), _p(g), _p(H))
    return float(mu[0]), g, H


def patches_for(blocks, free, w_inv=None, d=2):
    """Explicit patches of every moving DOF, in the reference's occurrence order."""
    from egg_b200 import wire

    blocks = [np.asarray(b) for b in blocks]
    N = free.shape[0]
    nc = 1 << d
    if w_inv is None:
        w_inv = np.eye(d)
    w_inv = np.asarray(w_inv, dtype=np.float64)
    uniform = w_inv.shape == (d, d)
    w0 = w_inv if uniform else w_inv[0]
    synth = bool(np.allclose(w0, w0[0, 0] * np.eye(d)) and (uniform or np.allclose(w_inv, w0)))
    interior = np.zeros(N, dtype=bool)
    if synth:
        for ids in blocks:
            if all(s >= 3 for s in ids.shape):
                interior[ids[tuple(slice(1, s - 1) for s in ids.shape)].reshape(-1)] = True
    Cc = wire.cell_corner_ids(blocks, d)
    ncell = Cc.shape[0]
    bits = wire.axis_bits(d)
    role_t = wire.role_table(d)
    b = np.arange(nc)
    sgn = np.where((b[:, None] & bits[None, :]) == 0, 1.0, -1.0)
    m_node = np.repeat(Cc[:, :, None], nc, axis=2).reshape(-1)
    m_cell = np.repeat(np.arange(ncell), nc * nc)
    m_b = np.tile(b, ncell * nc)
    m_role = np.tile(role_t.reshape(-1), ncell)
    keep = free[m_node]
    m_node, m_cell, m_b, m_role = m_node[keep], m_cell[keep], m_b[keep], m_role[keep]
    perm = np.argsort(m_node, kind="stable")
    m_node, m_cell, m_b, m_role = m_node[perm], m_cell[perm], m_b[perm], m_role[perm]
    dofs = np.flatnonzero(free).astype(np.int32)
    cnt = np.bincount(m_node, minlength=N)[dofs]
    off = np.concatenate([[0], np.cumsum(cnt)]).astype(np.int64)
    sid = m_cell * nc + m_b
    if uniform:
        W = np.broadcast_to(w_inv.reshape(1, d * d), (sid.size, d * d)).copy()
    else:
        W = w_inv.reshape(-1, d * d)[sid].copy()
    W[interior[m_node]] = np.eye(d).reshape(-1)
    out = {
        "dof": dofs,
        "off": off,
        "gc": Cc[m_cell, m_b].astype(np.int32),
        "role": m_role.astype(np.int32),
        "W": np.ascontiguousarray(W),
    }
    for k in range(d):
        out[f"gn{k}"] = Cc[m_cell, m_b ^ bits[k]].astype(np.int32)
        out[f"s{k}"] = sgn[m_b, k].copy()
    return out


def stencil_for(blocks, w_inv=None, d=2):
    from egg_b200 import wire

    _, gc, gn, s = wire.cell_stencil(blocks, d)
    if w_inv is None:
        w_inv = np.eye(d)
    w_inv = np.asarray(w_inv, dtype=np.float64)
    if w_inv.shape == (d, d):
        W, stride = w_inv.reshape(-1).copy(), 0
    else:
        W, stride = np.ascontiguousarray(w_inv.reshape(-1)), d * d
    out = {"gc": gc.astype(np.int32), "W": W, "stride": stride}
    for k in range(d):
        out[f"gn{k}"] = gn[k].astype(np.int32)
        out[f"s{k}"] = s[k]
    return out


def run(X, patches, stencil, n_sweeps, *, phase="barrier", delta=0.0, omega=1.0, report_every=0):
    """Block-Jacobi on a copy of X (N, 2); returns (X_out, energies, mindets)."""
    lib = load()
    Xw = np.ascontiguousarray(X, dtype=np.float64).reshape(-1).copy()
    k = report_every if report_every > 0 else max(n_sweeps, 1)
    nrep = (n_sweeps + k - 1) // k if n_sweeps > 0 else 0
    E = np.zeros(max(nrep, 1))
    M = np.zeros(max(nrep, 1))
    pt, st = patches, stencil
    r = lib.oracle_run2d(
        KIND[phase], float(delta), float(omega), int(n_sweeps), int(report_every), Xw.size // 2, _p(Xw),
        pt["dof"].size, _p(pt["dof"]), _p(pt["off"]), _p(pt["gc"]), _p(pt["gn0"]), _p(pt["gn1"]), _p(pt["s0"]),
        _p(pt["s1"]), _p(pt["role"]), _p(pt["W"]), None, st["gc"].size, _p(st["gc"]), _p(st["gn0"]),
        _p(st["gn1"]), _p(st["s0"]), _p(st["s1"]), _p(st["W"]), st["stride"], None, _p(E), _p(M))
    if r < 0:
        raise MemoryError("oracle_run2d: allocation failed")
    return Xw.reshape(-1, 2), E[:r], M[:r]


def run3(X, patches, stencil, n_sweeps, *, phase="barrier", delta=0.0, omega=1.0, report_every=0):
    """3D block-Jacobi on a copy of X (N, 3); returns (X_out, energies, mindets)."""
    lib = load()
    Xw = np.ascontiguousarray(X, dtype=np.float64).reshape(-1).copy()
    k = report_every if report_every > 0 else max(n_sweeps, 1)
    nrep = (n_sweeps + k - 1) // k if n_sweeps > 0 else 0
    E = np.zeros(max(nrep, 1))
    M = np.zeros(max(nrep, 1))
    pt, st = patches, stencil
    r = lib.oracle_run3d(
        KIND[phase], float(delta), float(omega), int(n_sweeps), int(report_every), Xw.size // 3, _p(Xw),
        pt["dof"].size, _p(pt["dof"]), _p(pt["off"]), _p(pt["gc"]), _p(pt["gn0"]), _p(pt["gn1"]), _p(pt["gn2"]),
        _p(pt["s0"]), _p(pt["s1"]), _p(pt["s2"]), _p(pt["role"]), _p(pt["W"]), st["gc"].size, _p(st["gc"]),
        _p(st["gn0"]), _p(st["gn1"]), _p(st["gn2"]), _p(st["s0"]), _p(st["s1"]), _p(st["s2"]), _p(st["W"]),
        st["stride"], _p(E), _p(M))
    if r < 0:
        raise MemoryError("oracle_run3d: allocation failed")
    return Xw.reshape(-1, 3), E[:r], M[:r]


def energy3(X, stencil, *, phase="barrier", delta=0.0):
    lib = load()
    Xw = np.ascontiguousarray(X, dtype=np.float64).reshape(-1)
    e, m = np.zeros(1), np.zeros(1)
    st = stencil
    lib.oracle_energy3d(KIND[phase], float(delta), _p(Xw), st["gc"].size, _p(st["gc"]), _p(st["gn0"]),
                        _p(st["gn1"]), _p(st["gn2"]), _p(st["s0"]), _p(st["s1"]), _p(st["s2"]), _p(st["W"]),
                        st["stride"], _p(e), _p(m))
    return float(e[0]), float(m[0])


def energy(X, stencil, *, phase="barrier", delta=0.0):
    lib = load()
    Xw = np.ascontiguousarray(X, dtype=np.float64).reshape(-1)
    e = np.zeros(1)
    m = np.zeros(1)
    st = stencil
    lib.oracle_energy2d(KIND[phase], float(delta), _p(Xw), st["gc"].size, _p(st["gc"]), _p(st["gn0"]),
                        _p(st["gn1"]), _p(st["s0"]), _p(st["s1"]), _p(st["W"]), st["stride"], None, _p(e), _p(m))
    return float(e[0]), float(m[0])


def ref_path(precision: str = "fp64") -> Path:
    return HERE / "_ref" / precision / f"cpp_core{sysconfig.get_config_var('EXT_SUFFIX')}"


def reference_root() -> Path | None:
    """The reference checkout that the recipes read: ``$EGG_REFERENCE_ROOT``, or
    a checkout named ``reference`` beside this repository.  None when neither
    holds the reference's ``src/bindings.cpp`` (the GPU hosts never have it;
    they use what was built here)."""
    env = os.environ.get("EGG_REFERENCE_ROOT")
    cand = Path(env) if env else HERE.parent.parent / "reference"
    return cand if (cand / "src" / "bindings.cpp").exists() else None


_ref_loaded: dict = {}


def load_ref(precision: str = "fp64"):
    """The reference core built from source (oracle/_ref), or None if absent:
    "fp64", "fp32", or "fp64snap" (fp64 with the shim's parallel loops run
    serially, shared-node refreshes before ghost fills: the race-free
    ordering of the reference's halo launch).

    Only one precision can be loaded per process (both builds are extension
    modules named ``cpp_core``); asking for the other one raises."""
    p = ref_path(precision)
    if not p.exists():
        return None
    if precision in _ref_loaded:
        return _ref_loaded[precision]
    if _ref_loaded:
        raise RuntimeError(f"reference core {list(_ref_loaded)[0]} already loaded; run {precision} in a new process")
    spec = importlib.util.spec_from_file_location("cpp_core", p)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    if bool(mod.REAL_IS_FLOAT) != (precision == "fp32"):
        raise RuntimeError(f"oracle/_ref/{precision} reports REAL_IS_FLOAT={mod.REAL_IS_FLOAT}")
    _ref_loaded[precision] = mod
    return mod
