"""Host-side drivers that sit above the session, mirroring the reference's
Python drivers for this path (``egg/smoothing/cpp_backend.py``).

* :func:`untangle` is the delta-continuation schedule of ``cpp_untangle``
  (``egg/smoothing/cpp_backend.py:773-848``): delta_0 = factor * |min det A|,
  ``sweeps_per_delta`` untangle sweeps per step, delta <- shrink * delta, until
  min det A > margin; the decision reads one min-det per step from the device.
"""

from __future__ import annotations

import numpy as np

__all__ = ["untangle", "structured_session"]


def structured_session(grid, *, w_inv=None, compact=False, precision=None, device="auto"):
    """CppStructuredSweepSession over a :class:`egg_b200.configs.Grid`."""
    from egg_b200 import cpp_core

    return cpp_core.CppStructuredSweepSession(
        grid.wire(w_inv=w_inv, compact=compact), grid.structured(), grid.X_flat(), device=device, dim=grid.d,
        precision=precision,
    )


def untangle(session, *, sweeps_per_delta=20, delta0_factor=2.0, shrink=0.8, max_outer=60, margin=1e-9,
             omega=0.5):
    """delta-continuation untangle on a resident session; returns
    (min det A, outer iterations, final delta)."""
    _e, md = session.energy("barrier")
    if md > margin:
        return float(md), 0, 0.0
    delta = delta0_factor * max(abs(md), 1e-12)
    outer = 0
    for _ in range(max_outer):
        _e, mds = session.run(sweeps_per_delta, phase="untangle", delta=delta, omega=omega)
        outer += 1
        md = float(np.asarray(mds)[-1])
        if md > margin:
            break
        delta *= shrink
    return float(md), outer, float(delta)
