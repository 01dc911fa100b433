"""The allocation-free energy entry point (egg_b200_session_energy_noalloc)
against egg_b200_session_energy on the same resident state."""

from __future__ import annotations

import numpy as np
import pytest

from tests.golden.gen_golden_fixtures import case_grid

pytestmark = pytest.mark.gpu

MAX_PARTIALS = 4096
CASES = ["disk_oh33", "square65s", "sphere_in_cube7", "cube9"]


def _session(core, name, precision="fp64"):
    g = case_grid(name)
    return core.CppStructuredSweepSession(g.wire(), g.structured(), g.X_flat(), dim=g.d, precision=precision)


@pytest.mark.parametrize("name", CASES)
def test_noalloc_matches_energy_on_two_calls(gpu, name):
    s = _session(gpu, name)
    for phase, delta in (("barrier", 0.0), ("shape_size", 0.0), ("untangle", 1e-3)):
        ref = s.energy(phase, delta)
        first = s.energy_noalloc(phase, delta)
        second = s.energy_noalloc(phase, delta)
        assert first == ref and second == ref, (phase, ref, first, second)
    s.run(3)
    ref = s.energy()
    assert s.energy_noalloc() == ref
    assert s.energy_noalloc() == ref


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_noalloc_partial_counts(gpu, precision):
    s = _session(gpu, "disk_oh33", precision)
    e, m = s.energy()
    for n in (1, 37, 148, MAX_PARTIALS, MAX_PARTIALS):
        en, mn = s.energy_noalloc(n_partials=n)
        assert abs(en - e) <= 1e-13 * abs(e), (n, en, e)
        assert mn == m


def test_noalloc_interleaved_sessions(gpu):
    """Calls made one after another from different sessions share the static
    array without carrying state from one to the next."""
    a, b = _session(gpu, "disk_oh33"), _session(gpu, "cube9")
    ra, rb = a.energy(), b.energy()
    for _ in range(2):
        assert a.energy_noalloc() == ra
        assert b.energy_noalloc() == rb


def test_noalloc_rejects_sizes_beyond_maximum(gpu):
    s = _session(gpu, "square65s")
    for n in (MAX_PARTIALS + 1, -1):
        with pytest.raises(ValueError, match="n_partials"):
            s.energy_noalloc(n_partials=n)
    assert s.energy_noalloc() == s.energy()


def test_noalloc_leaves_free_memory_unchanged(gpu):
    torch = pytest.importorskip("torch")
    s = _session(gpu, "disk_oh33")
    s.energy_noalloc()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(50):
        s.energy_noalloc()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
