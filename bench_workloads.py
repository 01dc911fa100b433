"""The other measured configurations of the structured TMOP path, run by
``python bench.py --workload NAME`` (one GPU; same JSON line as the default
4097^2 square):

  disk_oh65      5-block unit-disk O-H, 65^2 nodes per block, +-0.25h noise,
                 shape metric, 40 block-Jacobi sweeps per step, fp64
  untangle1025   1025^2 square with ~5% of cells inverted: delta-continuation
                 untangle (20 sweeps per delta) then shape+size with the
                 mean-size target, 1000 sweeps in total per step; fp64 and
                 mixed
  sphere129_fas  7-block sphere-in-cube, 129^3 nodes per block, +-0.2h noise,
                 FAS V(2,2) cycles with at most 4 levels, mixed; every DOF
                 relaxed at every level counts as one update
  batch256       256 independent 3-9 block meshes (block sides 17..257,
                 +-0.25h), 20-sweep chunks replayed from a CUDA graph, mixed;
                 plus one 64x64 (or smaller) control net per mesh solved
                 together by the reduced Gauss-Newton PCG

Inputs are seeded synthetic grids (numpy default_rng); the device time is
taken with CUDA events on the session stream.  The CPU baseline is the
reference core built from source (oracle/_ref, OpenMP on every host core)
on a bounded sample of the same workload.
"""

from __future__ import annotations

import os
import time

import numpy as np

UNIT = "vertex-updates/s"


def _timed(torch, s, local, fn, steps):
    """Device seconds of `steps` calls of fn, events on the session stream."""
    st = torch.cuda.ExternalStream(s.stream(), device=f"cuda:{local}")
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(st)
    for _ in range(steps):
        fn()
    b.record(st)
    b.synchronize()
    return a.elapsed_time(b) / 1e3


def _ref_rate(make_session, sweeps_per_call, free, target_s=10.0, **run_kw):
    """Reference-core updates/s: repeated run(sweeps) calls for ~target_s."""
    s = make_session()
    s.run(1, **run_kw)
    n, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < target_s:
        s.run(sweeps_per_call, **run_kw)
        n += sweeps_per_call
    dt = time.perf_counter() - t0
    return free * n / dt, n, dt


def _cpu(kind, sample, value):
    return {"value": value, "unit": UNIT, "cores": os.cpu_count(), "kind": kind, "sample": sample}


def _cpu_target(args, default: float) -> float:
    """Seconds of reference-core work per CPU baseline (shorter when the
    workload runs as a side configuration of the default bench)."""
    return float(getattr(args, "cpu_target_s", None) or default)


def _omp():
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))


def disk_oh65(torch, cpp_core, args, local):
    from egg_b200 import configs
    from oracle import oracle

    g = configs.disk_oh(65, frac=0.25, seed=0)
    s = cpp_core.CppStructuredSweepSession(g.wire(compact=True, device=f"cuda:{local}"), g.structured(), g.X_flat(),
                                           precision="fp64")
    s.autotune("barrier", 3)
    s.checkpoint()
    F = g.num_free

    def step():
        s.restore()
        s.run(40, report_every=20)

    for _ in range(args.warmup):
        step()
    s.reset_stats()
    dt = _timed(torch, s, local, step, args.steps)
    launches = s.launch_count()
    X0 = g.X_flat()
    s.set_X(X0)  # first transfer allocates the session's pinned staging: untimed
    s.get_X()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        s.set_X(X0)
        s.run(40, report_every=20)
        Xo = s.get_X()
    e2e = time.perf_counter() - t0
    line = {"workload": "disk_oh65", "value": F * 40 * args.steps / dt, "ms_per_step": 1e3 * dt / args.steps,
            "dtype": "f64", "gpu_launches": launches,
            "config": {"workload": "unit disk O-H, 5 blocks of 65^2, +-0.25h, shape, 40 sweeps per step",
                       "moving_dofs": F},
            "e2e": {"value": F * 40 * args.steps / e2e, "unit": UNIT, "h2d_bytes_per_step": int(X0.nbytes),
                    "d2h_bytes_per_step": int(Xo.nbytes) + 32}}
    ref = oracle.load_ref("fp64")
    if ref is not None and not args.no_cpu_baseline:
        _omp()
        r = ref.CppStructuredSweepSession(g.wire(), g.structured(), g.X_flat(), device="cpu")
        r.run(1)
        t0 = time.perf_counter()
        reps = 0
        while time.perf_counter() - t0 < _cpu_target(args, 5.0):
            r.run(40, report_every=20)
            reps += 1
        dt_r = time.perf_counter() - t0
        line["cpu_baseline"] = _cpu("reference", f"the full workload, {reps} x 40 sweeps in {dt_r:.1f} s",
                                    F * 40 * reps / dt_r)
    return line


def untangle1025(torch, cpp_core, args, local):
    from egg_b200 import configs, driver
    from oracle import oracle

    g = configs.tangled_square(1025, target=0.05, seed=0)
    F = g.num_free
    out = {}
    for prec in ("fp64", "mixed"):
        a = driver.structured_session(g, compact=True, precision=prec)
        a.autotune("untangle", 3)
        a.checkpoint()
        # shape+size session with the mean-size target (the mean signed corner
        # determinant hardly moves while interior nodes move inside the square)
        b = cpp_core.CppStructuredSweepSession(
            g.wire(compact=True, w_inv=configs.mean_size_w_inv(g.blocks, g.X)), g.structured(), g.X_flat(),
            precision=prec)
        # the autotuner times the resident data: tune the shape+size session on
        # an untangled state, which is what it sweeps (on the tangled start most
        # DOFs take the fp64 fallback and the timings say little)
        driver.untangle(a, sweeps_per_delta=20)
        b.set_X(a.get_X())
        b.autotune("shape_size", 3)

        def step():
            a.restore()
            md, outer, _ = driver.untangle(a, sweeps_per_delta=20)
            rest = 1000 - 20 * outer
            b.set_X(a.get_X())
            E, M = b.run(rest, phase="shape_size", report_every=rest)
            return md, outer, float(E[-1]), float(M[-1])

        step()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = [step() for _ in range(args.steps)]
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        md, outer, E, M = res[-1]
        out[prec] = {"seconds_per_step": dt / args.steps, "untangled": bool(md > 0), "delta_steps": outer,
                     "final_energy": E, "final_mindet": M, "value": F * 1000 * args.steps / dt,
                     "variants": {"untangle": a.variants()["variant"], "shape_size": b.variants()["variant"]}}
    rel = abs(out["mixed"]["final_energy"] - out["fp64"]["final_energy"]) / abs(out["fp64"]["final_energy"])
    line = {"workload": "untangle1025", "value": out["mixed"]["value"],
            "ms_per_step": 1e3 * out["mixed"]["seconds_per_step"], "dtype": "f32+f64",
            "config": {"workload": "1025^2 square, ~5% cells inverted, delta-continuation untangle then "
                                   "shape+size (mean-size target), 1000 sweeps per step", "moving_dofs": F},
            "fp64": out["fp64"], "mixed": out["mixed"],
            "mixed_vs_fp64": {"rel_energy": rel,
                              "same_untangle_status": out["mixed"]["untangled"] == out["fp64"]["untangled"],
                              "speedup": out["mixed"]["value"] / out["fp64"]["value"]},
            "timing": "wall clock per step with a device sync (the host decides each delta step)"}
    ref = oracle.load_ref("fp64")
    if ref is not None and not args.no_cpu_baseline:
        _omp()
        v, n, dt = _ref_rate(lambda: ref.CppStructuredSweepSession(g.wire(), g.structured(), g.X_flat(),
                                                                   device="cpu"),
                             5, F, target_s=_cpu_target(args, 10.0), phase="untangle", delta=1e-4, omega=0.5)
        line["cpu_baseline"] = _cpu("reference", f"untangle sweeps on the full grid, {n} sweeps in {dt:.1f} s", v)
    return line


def sphere129_fas(torch, cpp_core, args, local):
    from egg_b200 import configs
    from oracle import oracle

    n = int(os.environ.get("EGG_B200_SPHERE_N", "129"))
    g = configs.sphere_in_cube(n, frac=0.2, seed=0)
    s = cpp_core.CppStructuredSweepSession(g.wire(compact=True, device=f"cuda:{local}"), g.structured(), g.X_flat(),
                                           dim=3, precision="mixed")
    E0, M0 = s.energy()
    # the +-0.2h noise inverts a few thousand samples at the skewed shell
    # corners: untangle first (delta continuation), as the pipeline does
    from egg_b200 import driver

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    md_u, outer_u, _ = driver.untangle(s, sweeps_per_delta=20)
    torch.cuda.synchronize()
    t_untangle = time.perf_counter() - t0
    s.autotune("barrier", 3)
    s.checkpoint()
    E1, M1 = s.energy()
    cycles = 2

    def step():
        s.restore()
        return s.run_fas(cycles, nu_pre=2, nu_post=2, max_levels=4)

    for _ in range(max(1, args.warmup)):
        step()
    s.reset_stats()
    dt = _timed(torch, s, local, step, args.steps)
    upd = s.info()["updates"]
    launches = s.launch_count()
    E, M = step()
    # plain Jacobi sweeps on the same state: the sweep kernel's own rate
    s.restore()
    jac = _timed(torch, s, local, lambda: s.run(8, report_every=8), 1)
    line = {"workload": "sphere129_fas", "value": upd / dt, "ms_per_step": 1e3 * dt / args.steps,
            "dtype": "f32+f64", "gpu_launches": launches,
            "config": {"workload": f"sphere-in-cube, 7 blocks of {n}^3, +-0.2h, untangle, then FAS V(2,2) x "
                                   f"{cycles} per step, <= 4 levels", "moving_dofs": g.num_free,
                       "levels": s.mg_levels(), "updates_per_step": upd // args.steps},
            "untangle": {"seconds": t_untangle, "delta_steps": outer_u, "mindet_before": float(M0),
                         "mindet_after": float(md_u)},
            "energy": {"initial": float(E0), "after_untangle": float(E1), "after_step": [float(x) for x in E],
                       "mindet": float(M[-1])},
            "jacobi_updates_per_s": g.num_free * 8 / jac, "autotune": s.variants()}
    ref = oracle.load_ref("fp64")
    if ref is not None and not args.no_cpu_baseline:
        _omp()
        gs = configs.sphere_in_cube(33, frac=0.2, seed=0)
        v, nn, dt_r = _ref_rate(lambda: ref.CppStructuredSweepSession(gs.wire(), gs.structured(), gs.X_flat(),
                                                                      device="cpu", dim=3), 2, gs.num_free,
                              target_s=_cpu_target(args, 10.0))
        line["cpu_baseline"] = _cpu("reference", f"Jacobi sweeps on the 7 x 33^3 sphere-in-cube, {nn} sweeps in "
                                                 f"{dt_r:.1f} s", v)
    return line


def batch256(torch, cpp_core, args, local):
    from egg_b200 import configs, control
    from oracle import oracle

    nm = int(os.environ.get("EGG_B200_BATCH", "256"))
    ms = configs.batch_meshes(nm, seed=0)
    tup = [(g.wire(compact=True), g.structured(), g.X_flat()) for g in ms]
    wires = []
    for g in ms:
        b = int(np.argmax([blk.size for blk in g.blocks]))
        wires.append(control.control_wire(control.grid_block_nodes(g, b),
                                          tuple(min(64, n - 2) for n in g.blocks[b].shape), block=b))
    s = cpp_core.CppBatchSweepSession(tup, precision="mixed", control=wires)
    s.autotune("barrier", 3)
    s.checkpoint()
    F = sum(g.num_free for g in ms)

    def step():
        s.restore()
        s.run(20, report_every=20)

    for _ in range(args.warmup):
        step()
    s.reset_stats()
    dt = _timed(torch, s, local, step, args.steps)
    launches = s.launch_count()
    s.restore()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    reps = s.run_control(5)
    torch.cuda.synchronize()
    t_ctl = time.perf_counter() - t0
    line = {"workload": "batch256", "value": F * 20 * args.steps / dt, "ms_per_step": 1e3 * dt / args.steps,
            "dtype": "f32+f64", "gpu_launches": launches,
            "config": {"workload": f"{nm} meshes of 3-9 blocks (sides 17..257), +-0.25h, shape, one 20-sweep "
                                   "graph chunk per step", "moving_dofs": F, "nodes": sum(g.num_nodes for g in ms)},
            "control": {"outer_iterations": 5, "seconds": t_ctl,
                        "nets": nm, "free_controls": int(sum(w["free_idx"].size for w in wires)),
                        "mean_energy_drop": float(np.mean([r["energies"][0] - r["energies"][-1] for r in reps])),
                        "mean_pcg_iters": float(np.mean([np.mean(r["pcg_iters"]) if len(r["pcg_iters"]) else 0
                                                         for r in reps]))}}
    ref = oracle.load_ref("fp64")
    if ref is not None and not args.no_cpu_baseline:
        _omp()
        sample = ms[:16] if _cpu_target(args, 10.0) >= 10.0 else ms[:4]
        t0 = time.perf_counter()
        for g in sample:
            r = ref.CppStructuredSweepSession(g.wire(), g.structured(), g.X_flat(), device="cpu")
            r.run(20, report_every=20)
        dt_r = time.perf_counter() - t0
        line["cpu_baseline"] = _cpu("reference", f"the first {len(sample)} meshes, one session and 20 sweeps each, "
                                                 f"{dt_r:.1f} s (session build included)",
                                    sum(g.num_free for g in sample) * 20 / dt_r)
    return line


WORKLOADS = {"disk_oh65": disk_oh65, "untangle1025": untangle1025, "sphere129_fas": sphere129_fas,
             "batch256": batch256}
