"""The C-ABI library and the pybind surface: symbols, errors, host-side
validation (runs without a GPU; nothing here launches a kernel)."""

from __future__ import annotations

import ctypes
import re

import numpy as np
import pytest

from egg_b200 import configs, lib_path
from tests.conftest import ROOT, gpu_available


def _declared_functions():
    text = (ROOT / "include" / "egg_b200.h").read_text()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(egg_b200_\w+)\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(lib_path()))
    names = _declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    lib.egg_b200_abi_version.restype = ctypes.c_int
    assert lib.egg_b200_abi_version() == 1


def test_cpp_core_surface(core):
    assert core.ping() == 0
    assert core.REAL_IS_FLOAT in (True, False)
    for m in ("run", "run_fas", "mg_levels", "get_X", "run_control", "get_C", "set_C"):
        assert hasattr(core.CppStructuredSweepSession, m)
    for f in ("cpp_structured_sweep", "metric_eval", "metric_eval_3d", "patch_eval", "newton_step", "energy_mindet",
              "directional_eval", "geometry_project", "geometry_project_batch", "geometry_tangent"):
        assert hasattr(core, f)


def test_cpp_core_covers_the_reference_module_surface(core):
    """Every public name of the reference's cpp_core module (built from its
    sources into oracle/_ref) exists here, with the same keyword names."""
    import json
    import subprocess
    import sys

    from oracle import oracle

    if not oracle.ref_path("fp64").exists():
        pytest.skip("oracle/_ref not built in this environment")
    code = ("import json,sys,inspect; sys.path.insert(0, %r); from oracle import oracle; m = oracle.load_ref('fp64');"
            "print(json.dumps({n: getattr(m, n).__doc__ or '' for n in dir(m) if not n.startswith('_')}))"
            % str(oracle.HERE.parent))
    out = subprocess.run([sys.executable, "-c", code], check=True, capture_output=True, text=True).stdout
    ref = json.loads(out.strip().splitlines()[-1])
    missing = [n for n in ref if not hasattr(core, n)]
    assert not missing, missing
    for cls in ("CppStructuredSweepSession",):
        assert hasattr(core, cls)


def _inputs(n=9):
    g = configs.unit_square(n, frac=0.2, seed=0)
    return g, g.wire(), g.structured(), g.X_flat()


def test_cpu_device_is_refused(core):
    g, ctx, st, X = _inputs()
    with pytest.raises(RuntimeError, match="GPU only"):
        core.CppStructuredSweepSession(ctx, st, X, device="cpu")


@pytest.mark.skipif(gpu_available(), reason="a GPU is present")
def test_no_device_raises_runtime_error(core):
    g, ctx, st, X = _inputs()
    with pytest.raises(RuntimeError, match="no CUDA device"):
        core.CppStructuredSweepSession(ctx, st, X)


def _expect_value_error(core, ctx, st, X, match, dim=2):
    with pytest.raises(ValueError, match=match):
        core.CppStructuredSweepSession(ctx, st, X, dim=dim)


def test_malformed_contexts_raise_value_error(core):
    """Mirrors the reference's validate_context checks (src/bindings.cpp:98-252)."""
    g, ctx, st, X = _inputs()
    _expect_value_error(core, ctx, st, X.reshape(-1, 2), "flat 1-D")
    _expect_value_error(core, ctx, st, X[:-1], "multiple of d")
    _expect_value_error(core, ctx, st, X, "dimension must be 2 or 3", dim=4)

    d = g.disk = configs.disk_oh(9)
    ctx, st, X = d.wire(), d.structured(), d.X_flat()
    grp = ctx["groups"][0]
    bad = {**ctx, "groups": [{**grp, "P_of": grp["P_of"] + 1}]}
    _expect_value_error(core, bad, st, X, "sum\\(P_of\\)")
    gc = grp["gc"].copy()
    gc[0] = 10**6
    _expect_value_error(core, {**ctx, "groups": [{**grp, "gc": gc}]}, st, X, "gc index")
    role = grp["role"].copy()
    role[0] = 7
    _expect_value_error(core, {**ctx, "groups": [{**grp, "role": role}]}, st, X, "role 7 out of range")
    dofs = grp["dof_idx"].copy()
    dofs[0] = -3
    _expect_value_error(core, {**ctx, "groups": [{**grp, "dof_idx": dofs}]}, st, X, "dof_idx index")
    ent = {"free": {**grp["entities"]["free"], "dof_local": grp["entities"]["free"]["dof_local"][1:]}}
    _expect_value_error(core, {**ctx, "groups": [{**grp, "entities": ent}]}, st, X, "not covered")
    es = dict(ctx["energy_stencil"])
    es["gn0"] = es["gn0"][:-1]
    _expect_value_error(core, {**ctx, "energy_stencil": es}, st, X, "energy_stencil gn")
    bgd = list(st["block_global_dof"])
    bgd[0] = bgd[0][:-1]
    _expect_value_error(core, ctx, {**st, "block_global_dof": bgd}, X, "block_global_dof length")
    W = grp["W_inv"]
    _expect_value_error(core, {**ctx, "groups": [{**grp, "W_inv": np.zeros(5)}]}, st, X, "W_inv")
    il = grp["interior_logical"].copy()
    k = int(np.flatnonzero(grp["interior_block"] >= 0)[0])
    il[k] = [0, 0]
    _expect_value_error(core, {**ctx, "groups": [{**grp, "interior_logical": il}]}, st, X, "not strictly interior")
    assert W.shape == (1, 4)


def test_constrained_dofs_are_rejected(core):
    g, ctx, st, X = _inputs()
    grp = ctx["groups"][0]
    ent = {"line": {"tag": 1, "kFields": 4, "dof_local": grp["entities"]["free"]["dof_local"],
                    "records": np.zeros(4 * grp["D"])}}
    with pytest.raises((NotImplementedError, RuntimeError)):
        core.CppStructuredSweepSession({**ctx, "groups": [{**grp, "entities": ent}]}, st, X)


def test_energy_stencil_checks_on_many_threads_report_the_first_bad_sample(core):
    """The reference-form stencil is validated on host threads over sample
    slices (257^2: 262,144 samples, several slices); a bad index in a late
    slice is still found, and with two bad samples the earlier one is
    reported, as a serial scan would (src/bindings.cpp:98-252 messages)."""
    g = configs.unit_square(257, frac=0.2, seed=0)
    ctx, st, X = g.wire(), g.structured(), g.X_flat()
    es = ctx["energy_stencil"]
    ns = es["num_samples"]
    gn1 = es["gn1"].copy()
    gn1[ns - 3] = g.num_nodes + 5
    _expect_value_error(core, {**ctx, "energy_stencil": {**es, "gn1": gn1}}, st, X, f"index {g.num_nodes + 5} out")
    gc = es["gc"].copy()
    gc[ns // 3] = -7
    _expect_value_error(core, {**ctx, "energy_stencil": {**es, "gn1": gn1, "gc": gc}}, st, X, "index -7 out")
