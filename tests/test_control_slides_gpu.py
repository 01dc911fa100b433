"""Topologies with sliding-wall frames, exercised by the reference's tests.

tests/golden/ref_dropin_slides.pkl.gz holds every call that three of the
reference's multi-block driver tests (``tests/smoothing/
test_control_topo_cpp.py``: ``test_device_sliding_wall_roots``,
``test_single_block_segmented_wall``, ``test_device_3d_two_block_run``) made
on ``egg._cpp.cpp_core``: a two-block seam whose bottom rides a line segment
(then the same grid with fixed walls), a single block whose bottom rides a
cubic B-spline, and a rotated 3D two-block slab.  The sliding runs rebuild
their frame every outer iteration (root reprojection, member move, wall b
re-extension, db/dC model) and report each frame's energy jump; the
driver's own entity projections (``geometry_project_batch``) are replayed
too.  Recorded by ``tests/golden/gen_dropin_trace.py --slides``.
"""

from __future__ import annotations

import pytest

from tests import control_replay

pytestmark = pytest.mark.gpu

_EVENTS = control_replay.load("ref_dropin_slides.pkl.gz")
SCENARIOS = sorted({ev["scenario"] for ev in _EVENTS})


# The B-spline wall's feet come from Newton iterations that round with each
# compiler's FMA contraction (the entity tests hold them to 1e-10): the
# lattice then agrees to ~1e-11 and the min det, a minimum over the samples
# next to the wall, to ~1e-8 relative; energies and frame jumps to ~1e-14.
_TOL = {"bspline_block": (1e-7, 1e-10)}


@pytest.mark.parametrize("scenario", SCENARIOS)
def test_reference_sliding_topology_replay(gpu, scenario):
    rtol, x_atol = _TOL.get(scenario, (control_replay.RTOL, 1e-10))
    assert control_replay.replay(gpu, _EVENTS, scenario, rtol=rtol, x_atol=x_atol) > 0
