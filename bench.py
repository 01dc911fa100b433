"""Benchmark: vertex Newton updates/s of the structured TMOP sweep on B200.

Workload (one "step"): 200 block-Jacobi sweeps of the TMOP shape metric on a
single 4097 x 4097 block of the unit square whose interior nodes carry seeded
+-0.3 h uniform noise (16.77 M moving DOFs), starting every step from the same
positions.  `value` is device-resident throughput (moving DOFs x sweeps / s)
with the fp32-bulk / fp64-guarded ("mixed") sweep; `e2e` is the same step
through the public API (set_X from host memory, run, get_X back to host); the
plain-fp64 sweep is reported beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun (N > 1) every rank runs an independent replica (the path has no
cross-GPU exchange); value = all ranks' updates / max-over-ranks time.
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_SIDE = 4097
FRAC = 0.3
SEED = 0
SWEEPS = 200
METRIC = "vertex Newton updates/s"
UNIT = "vertex-updates/s"
# Algorithmic bytes per moving-DOF update of the fused sweep: read the node's
# fp64 position once, write it once (neighbours are reused through shared
# memory; structure is synthesized, not read).
BYTES_PER_UPDATE = 2 * 2 * 8
# DRAM bytes (read + write) and thread instructions per moving-DOF update of
# the mixed interior kernel (interior_x2_kernel<8,16,7>), from one ncu capture
# of a 2049^2 launch (4,190,209 DOFs; the store exceeds L2): traffic and
# instructions grow in proportion to the DOFs swept.
DRAM_BYTES_PER_UPDATE = 527.0e6 / 16769025
INSTR_PER_UPDATE = 1248.0
# Issue roof: 148 SMs x 4 schedulers x 32 lanes, one warp instruction per
# scheduler per cycle.
ISSUE_LANES = 148 * 4 * 32


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """Samples SM clock and throttle reasons through NVML while running."""

    def __init__(self, index: int, period: float = 0.1):
        self.index, self.period = index, period
        self.samples = []
        self._stop = threading.Event()
        self._t = None
        self.ok = False

    def __enter__(self):
        try:
            import pynvml

            pynvml.nvmlInit()
            self._nv = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
            self.ok = True
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        except Exception:  # noqa: BLE001 - clocks are advisory when NVML is absent
            self.ok = False
        return self

    def _run(self):
        nv = self._nv
        while not self._stop.is_set():
            try:
                mhz = nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM)
                reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                self.samples.append((mhz, reasons))
            except Exception:  # noqa: BLE001
                pass
            self._stop.wait(self.period)

    def __exit__(self, *exc):
        self._stop.set()
        if self._t:
            self._t.join()

    def summary(self):
        if not self.ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml unavailable"]}
        nv = self._nv
        names = {
            "gpu_idle": nv.nvmlClocksEventReasonGpuIdle,
            "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap,
            "hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
            "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
            "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
            "hw_power_brake": nv.nvmlClocksEventReasonHwPowerBrakeSlowdown,
        }
        seen = set()
        for _, r in self.samples:
            for k, bit in names.items():
                if r & bit:
                    seen.add(k)
        mhz = [m for m, _ in self.samples]
        return {"sm_mhz": float(np.median(mhz)), "sm_max_mhz": float(self.max_mhz), "reasons": sorted(seen),
                "samples": len(mhz)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _pg_init(ws, backend):
    if ws <= 1:
        return None
    import datetime

    import torch.distributed as dist

    dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
    return dist


def _max_over_ranks(dist, x, device=None):
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(dist, updates_per_rank, dt_local, device=None):
    """Whole-job updates/s of N independent replicas: every rank's updates
    over the slowest rank's time (max over ranks). Returns (value, dt_max)."""
    ws = dist.get_world_size() if dist is not None else 1
    dt = _max_over_ranks(dist, dt_local, device=device)
    return ws * updates_per_rank / dt, dt


def _barrier(dist):
    if dist is not None:
        dist.barrier()


def _grid(n=N_SIDE):
    from egg_b200 import configs

    return configs.unit_square(n, frac=FRAC, seed=SEED)


def cpu_baseline(threads=None, target_s=12.0):
    """The reference core (oracle/_ref, OpenMP) on a bounded sample of the
    workload: a 1025^2 block with the same noise, timed sweeps after warm-up."""
    from egg_b200 import configs
    from oracle import oracle

    ref = oracle.load_ref("fp64")
    cores = threads or os.cpu_count()
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    g = configs.unit_square(1025, frac=FRAC, seed=SEED)
    if ref is not None:
        s = ref.CppStructuredSweepSession(g.wire(), g.structured(), g.X_flat(), device="cpu")
        s.run(1)
        t0 = time.perf_counter()
        n = 0
        while time.perf_counter() - t0 < target_s:
            s.run(2)
            n += 2
        dt = time.perf_counter() - t0
        kind = "reference"
    else:
        pt, sc = oracle.patches_for(g.blocks, g.free), oracle.stencil_for(g.blocks)
        oracle.run(g.X, pt, sc, 1)
        t0 = time.perf_counter()
        n = 0
        X = g.X
        while time.perf_counter() - t0 < target_s:
            X, _, _ = oracle.run(X, pt, sc, 1)
            n += 1
        dt = time.perf_counter() - t0
        kind, cores = "port", 1
    return {"value": g.num_free * n / dt, "unit": UNIT, "cores": int(cores), "kind": kind,
            "sample": f"1025x1025 unit square, +-0.3h noise, shape metric, {n} sweeps in {dt:.1f} s"}


def _first_at(E, target, tol):
    """1-based index of the first report at or below target (1 + tol)
    relative, or None."""
    hit = np.nonzero(np.asarray(E) <= target + tol * abs(target))[0]
    return int(hit[0]) + 1 if len(hit) else None


def time_to_energy_tol(torch, cpp_core, local, sessions, sweeps, tol=1e-6, fas_cycles=60, every=10, cpu=True):
    """Time to the job's energy: how long block-Jacobi and FAS V(2,2), in
    both precisions, take to bring the energy within tol (relative) of the
    energy the plain fp64 sweep reaches after the job's `sweeps` sweeps.

    A converged energy is not a usable target on this workload: the barrier
    never lets a DOF next to one of its ~2k inverted samples move, and those
    samples dominate the energy, so both solvers keep creeping (the reported
    `fas_last_cycle_change_rel` after `fas_cycles` cycles shows how much).
    The target is therefore e_T = E_fp64(`sweeps` Jacobi sweeps).  Each solver
    is traced (Jacobi with a report every `every` sweeps up to `sweeps` + 2
    reports, FAS per cycle up to `fas_cycles`); k is the first report at or
    below e_T (1 + tol), and its k steps from the start are then timed on the
    device.  With cpu=True the reference core (oracle/_ref, all host cores)
    times FAS to the same kind of target on a 1025^2 sample of the workload.
    """
    from egg_b200 import configs

    def fas(s, k):
        return s.run_fas(k, nu_pre=2, nu_post=2)

    def jac(s, k):
        return s.run(k)

    def timed(s, fn, k):
        stream = torch.cuda.ExternalStream(s.stream(), device=f"cuda:{local}")
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.restore()
        torch.cuda.synchronize()
        ev0.record(stream)
        E, _ = fn(s, k)
        ev1.record(stream)
        ev1.synchronize()
        return ev0.elapsed_time(ev1) / 1e3, float(E[-1])

    def measure(ss):
        ss["fp64"].restore()
        e_T = float(ss["fp64"].run(sweeps)[0][-1])
        res = {"target_energy": e_T, "target": f"fp64 energy after {sweeps} Jacobi sweeps",
               "jacobi": {"sweeps": {}, "seconds": {}}, "fas": {"cycles": {}, "seconds": {}}}
        for prec, s in ss.items():
            s.restore()
            E, _ = s.run(sweeps + 2 * every, report_every=every)
            k = _first_at(E, e_T, tol)
            res["jacobi"]["sweeps"][prec] = None if k is None else every * k
            if k is not None:
                res["jacobi"]["seconds"][prec] = timed(s, jac, every * k)[0]
            s.restore()
            E, _ = fas(s, fas_cycles)
            if prec == "fp64":
                res["fas_last_cycle_change_rel"] = abs(float(E[-1] - E[-2])) / abs(float(E[-1]))
            k = _first_at(E, e_T, tol)
            res["fas"]["cycles"][prec] = k
            if k is not None:
                res["fas"]["seconds"][prec] = timed(s, fas, k)[0]
        return res

    out = {"tol_rel": tol, "square4097": measure(sessions)}
    g = configs.unit_square(1025, frac=FRAC, seed=SEED)
    small = {}
    for prec in ("fp64", "mixed"):
        s = cpp_core.CppStructuredSweepSession(g.wire(compact=True), g.structured(), g.X_flat(),
                                               device=f"cuda:{local}", precision=prec)
        s.autotune("barrier", 3)
        s.checkpoint()
        small[prec] = s
    r = measure(small)
    from oracle import oracle

    ref = oracle.load_ref("fp64") if cpu else None
    k = r["fas"]["cycles"].get("fp64")
    if ref is not None and k is not None:
        os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
        rs = ref.CppStructuredSweepSession(g.wire(), g.structured(), g.X_flat(), device="cpu")
        t0 = time.perf_counter()
        E_ref, _ = rs.run_fas(k, nu_pre=2, nu_post=2)
        r["fas"]["seconds"]["reference_cpu"] = time.perf_counter() - t0
        r["fas"]["reference_cpu_energy_at_k"] = float(E_ref[-1])
        r["fas"]["reference_cpu_cores"] = os.cpu_count()
    out["square1025"] = r
    return out


def _error_stats(X, E, M, Xr, Er, Mr, h):
    """The north star's error figures of a result against an fp64 oracle."""
    return {"max_dx_over_h": float(np.abs(np.asarray(X) - np.asarray(Xr)).max() / h),
            "rel_energy": abs(float(E) - float(Er)) / abs(float(Er)),
            "mindet": float(M), "mindet_oracle": float(Mr),
            "same_untangle_status": bool((float(M) > 0) == (float(Mr) > 0))}


def error_vs_fp64_oracle(g, sessions, sweeps, cpu=True, ref_sweeps=2):
    """Errors of both GPU paths against fp64 oracles on the bench grid.

    * reference_core: `ref_sweeps` sweeps from the start positions by the
      reference core itself (oracle/_ref, fp64), against the same sweeps on
      each GPU path;
    * gpu_fp64: the mixed path after the job's `sweeps` sweeps against the
      plain fp64 GPU path (pinned to the reference core on every parity case).
    h is the grid's nominal spacing.
    """
    h = 1.0 / (int(round(np.sqrt(g.num_nodes))) - 1)
    out = {"h": h}
    runs = {}
    for prec, s in sessions.items():
        s.restore()
        E, M = s.run(sweeps)
        runs[prec] = (s.get_X(), float(E[-1]), float(M[-1]))
    Xf, Ef, Mf = runs["fp64"]
    Xm, Em, Mm = runs["mixed"]
    out["gpu_fp64"] = {"sweeps": sweeps, "mixed": _error_stats(Xm, Em, Mm, Xf, Ef, Mf, h)}
    if cpu:
        from oracle import oracle

        ref = oracle.load_ref("fp64")
        if ref is not None:
            os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
            Xr, Er, Mr = ref.cpp_structured_sweep(g.wire(), g.structured(), g.X_flat(), ref_sweeps, device="cpu",
                                                  phase="barrier", report_every=ref_sweeps)
            res = {"sweeps": ref_sweeps, "cores": os.cpu_count()}
            for prec, s in sessions.items():
                s.restore()
                E, M = s.run(ref_sweeps)
                res[prec] = _error_stats(s.get_X(), E[-1], M[-1], Xr, Er[-1], Mr[-1], h)
            out["reference_core"] = res
    return out


def run_reference(args):
    """--impl reference: the reference's own CPU implementation, all host threads."""
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    from oracle import oracle

    ref = oracle.load_ref("fp64")
    if ref is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (reference core built from source) missing"}))
        return 0
    cores = os.cpu_count()
    os.environ["OMP_NUM_THREADS"] = str(cores)
    g = _grid()
    t0 = time.perf_counter()
    s = ref.CppStructuredSweepSession(g.wire(), g.structured(), g.X_flat(), device="cpu")
    setup = time.perf_counter() - t0
    per_step = int(os.environ.get("EGG_B200_REF_SWEEPS", "2"))
    for _ in range(args.warmup):
        s.run(per_step)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        s.run(per_step)
        times.append(time.perf_counter() - t0)
    ms = 1e3 * float(np.mean(times))
    value = g.num_free * per_step / (ms / 1e3)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{N_SIDE}x{N_SIDE} unit square, +-0.3h seeded noise, TMOP shape, "
                               f"{per_step} block-Jacobi sweeps per step (bounded sample of the 200-sweep job)",
                   "moving_dofs": g.num_free, "setup_s": setup},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"{per_step} sweeps per step on the full {N_SIDE}^2 grid"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_workload(args):
    """One of the other measured configurations (bench_workloads.py), one GPU."""
    import torch

    import bench_workloads
    from egg_b200 import cpp_core

    ws, rank, local = _dist()
    if ws > 1:
        if rank == 0:
            print(json.dumps({"workload": args.workload, "unavailable": "the extra workloads run on one GPU"}))
        return 0
    fn = bench_workloads.WORKLOADS[args.workload]
    torch.cuda.set_device(local)
    with ClockSampler(local) as clk:
        line = fn(torch, cpp_core, args, local)
    out = {"metric": METRIC, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "data": "synthetic"}
    out.update(line)
    out["clocks"] = clk.summary()
    print(json.dumps(out))
    return 0


def side_configs(args, local):
    """The other benchmark configurations (bench_workloads.py: the 5-block
    disk, the 1025^2 untangle, the 7-block sphere FAS, the 256-mesh batch),
    each on a short sample -- at most 2 timed steps after 1 warm-up, bounded
    reference-core samples -- so the default run reports every configuration.
    A failing configuration reports its error instead of a value."""
    import types

    import torch

    import bench_workloads
    from egg_b200 import cpp_core

    sub = types.SimpleNamespace(steps=max(1, min(args.steps, 2)), warmup=1, no_cpu_baseline=args.no_cpu_baseline,
                                cpu_target_s=3.0)
    out = {}
    for name, fn in bench_workloads.WORKLOADS.items():
        t0 = time.perf_counter()
        try:
            with ClockSampler(local) as clk:
                line = fn(torch, cpp_core, sub, local)
            line["clocks"] = clk.summary()
            line["steps"], line["warmup"] = sub.steps, sub.warmup
        except Exception as exc:  # reported in the line, the headline stands
            line = {"workload": name, "error": f"{type(exc).__name__}: {exc}"}
        line["wall_s"] = time.perf_counter() - t0
        out[name] = line
        torch.cuda.empty_cache()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="egg_b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sweeps", type=int, default=SWEEPS)
    ap.add_argument("--only", choices=["fp64", "mixed"], default=None,
                    help="time one precision only and skip e2e (profiling runs)")
    ap.add_argument("--n", type=int, default=N_SIDE, help="grid side (profiling runs)")
    ap.add_argument("--variant", type=int, default=None,
                    help="pin the interior-kernel variant instead of autotuning (profiling runs)")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other configurations' short samples in the default line")
    ap.add_argument("--workload", default="square4097",
                    help="square4097 (default), disk_oh65, untangle1025, sphere129_fas, batch256")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload != "square4097":
        return run_workload(args)

    ws, rank, local = _dist()
    import torch

    torch.cuda.set_device(local)
    dist = _pg_init(ws, "nccl")
    from egg_b200 import cpp_core

    g = _grid(args.n)
    t_setup = time.perf_counter()
    g.wire(compact=True)
    st = g.structured()
    setup = {"wire_host_s": time.perf_counter() - t_setup}
    # The same wire from the device builder (the session below uses it), and
    # the reference-form wire with the energy stencil's per-sample arrays.
    # Best of three builds each: a single build can catch a host-side stall
    # (page reclaim) of several hundred ms.
    dev = f"cuda:{local}"
    g.wire(compact=True, device=dev)  # first call pays the context's lazy module load
    best = []
    for _ in range(3):
        t_setup = time.perf_counter()
        ctx = g.wire(compact=True, device=dev)
        best.append(time.perf_counter() - t_setup)
    setup["wire_device_s"] = min(best)
    best = []
    for _ in range(3):
        t_setup = time.perf_counter()
        full = g.wire(device=dev)
        best.append(time.perf_counter() - t_setup)
        nbytes = int(sum(v.nbytes for v in full["energy_stencil"].values() if isinstance(v, np.ndarray))
                     + sum(v.nbytes for v in full["groups"][0].values() if isinstance(v, np.ndarray)))
        del full
    setup["wire_full_device_s"] = min(best)
    setup["wire_full_bytes"] = nbytes
    X0 = g.X_flat()
    F = g.num_free
    sweeps = args.sweeps
    results = {}
    for prec in ([args.only] if args.only else ["fp64", "mixed"]):
        t_setup = time.perf_counter()
        s = cpp_core.CppStructuredSweepSession(ctx, st, X0, device=f"cuda:{local}", precision=prec)
        setup[f"session_create_{prec}_s"] = time.perf_counter() - t_setup
        if args.variant is None:
            s.autotune("barrier", 3)
        else:
            s.set_variant(args.variant)
        s.checkpoint()
        for _ in range(args.warmup):
            s.restore()
            s.run(sweeps)
        s.reset_stats()
        s.set_profiling(prec == "mixed")
        # Device time on the session's own stream, where every kernel of the
        # step is issued (torch's current stream would not see them).
        stream = torch.cuda.ExternalStream(s.stream(), device=f"cuda:{local}")
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        _barrier(dist)
        torch.cuda.synchronize()
        with ClockSampler(local) as clk:
            ev0.record(stream)
            E = None
            for _ in range(args.steps):
                s.restore()
                E, M = s.run(sweeps)
            ev1.record(stream)
            ev1.synchronize()
            torch.cuda.synchronize()
        dt = ev0.elapsed_time(ev1) / 1e3
        launches = s.launch_count()
        stats = s.kernel_stats()
        s.set_profiling(False)
        _v, dt = replica_throughput(dist, F * sweeps * args.steps, dt, device=f"cuda:{local}")
        results[prec] = {"dt": dt, "E": float(E[-1]), "M": float(M[-1]), "stats": stats, "launches": launches,
                         "clocks": clk.summary(), "session": s, "variants": s.variants()}

    if args.only:
        r = results[args.only]
        if rank == 0:
            print(json.dumps({"only": args.only, "n": args.n, "sweeps": sweeps, "steps": args.steps,
                              "variants": r["variants"], "ms_per_step": 1e3 * r["dt"] / args.steps,
                              "value": ws * F * sweeps * args.steps / r["dt"], "E": r["E"], "M": r["M"]}))
        if dist is not None:
            dist.destroy_process_group()
        return 0
    mixed = results["mixed"]
    ms_step = 1e3 * mixed["dt"] / args.steps
    value = ws * F * sweeps * args.steps / mixed["dt"]
    v64 = ws * F * sweeps * args.steps / results["fp64"]["dt"]

    # e2e through the public API with host buffers (mixed precision).  The
    # step's input sits in page-locked host memory -- a get_X result, which
    # the core hands out from its pinned pool -- so set_X and get_X are one
    # DMA each.
    s = mixed["session"]
    s.set_X(np.ascontiguousarray(X0))
    Xh = s.get_X()
    assert np.array_equal(Xh, X0)
    s.set_X(Xh)
    s.run(sweeps)
    warm = [s.get_X(), s.get_X()]  # warm-up: the loop below holds one result while fetching the next
    del warm
    _barrier(dist)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        s.set_X(Xh)
        _e, _m = s.run(sweeps)
        Xout = s.get_X()
    e2e_value, e2e_dt = replica_throughput(dist, F * sweeps * args.steps, time.perf_counter() - t0,
                                           device=f"cuda:{local}")

    tte = err = None
    if ws == 1:
        sess = {p: results[p]["session"] for p in ("fp64", "mixed")}
        err = error_vs_fp64_oracle(g, sess, sweeps, cpu=not args.no_cpu_baseline)
        tte = time_to_energy_tol(torch, cpp_core, local, sess, sweeps, cpu=not args.no_cpu_baseline)

    # Roofline of the dominant kernel (interior sweep), from the live events.
    k_ms, k_n = mixed["stats"]["interior_sweep"]
    hbm, peak_kind = _peaks()
    avg_ms = k_ms / max(k_n, 1)
    achieved = BYTES_PER_UPDATE * F / (avg_ms / 1e3) / 1e9
    roof = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
            "traffic": DRAM_BYTES_PER_UPDATE * F, "traffic_unit": "bytes per launch (ncu dram read+write)",
            "algorithmic_bytes": BYTES_PER_UPDATE * F, "kernel": "interior_x2_kernel (mixed)",
            "avg_launch_ms": avg_ms, "peak_source": peak_kind,
            "note": "frac states HBM use; the binding roof is instruction issue (see issue)"}
    mhz = mixed["clocks"].get("sm_mhz") or 1965.0
    upd_rate = F / (avg_ms / 1e3)
    roof["issue"] = {"thread_instructions_per_update": INSTR_PER_UPDATE,
                     "achieved": INSTR_PER_UPDATE * upd_rate, "peak": ISSUE_LANES * mhz * 1e6,
                     "unit": "thread instructions/s", "frac": INSTR_PER_UPDATE * upd_rate / (ISSUE_LANES * mhz * 1e6),
                     "sm_mhz": mhz, "source": "instructions per update from ncu (profiles/), rate from live events"}
    total_ms = sum(v[0] for v in mixed["stats"].values())
    share = {k: v[0] / total_ms for k, v in mixed["stats"].items() if v[1]}

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": f"{N_SIDE}x{N_SIDE} unit square single block, +-0.3h seeded noise, TMOP shape, "
                               f"{sweeps} block-Jacobi sweeps per step, omega=1",
                   "moving_dofs": F, "parallelism": "replicas" if ws > 1 else "single-gpu",
                   "l2": "inputs (269 MB fp64 store x2) larger than L2"},
        "fp64": {"value": v64, "ms_per_step": 1e3 * results["fp64"]["dt"] / args.steps,
                 "final_energy": results["fp64"]["E"], "final_mindet": results["fp64"]["M"]},
        "mixed": {"final_energy": mixed["E"], "final_mindet": mixed["M"],
                  "rel_energy_vs_fp64": abs(mixed["E"] - results["fp64"]["E"]) / abs(results["fp64"]["E"]),
                  "speedup_vs_fp64": value / v64},
        "roofline": roof, "kernel_share": share,
        "autotune": {"mixed": mixed["variants"], "fp64": results["fp64"]["variants"]},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(X0.nbytes),
                "d2h_bytes_per_step": int(Xout.nbytes + 16)},
        "gpu_launches": int(mixed["launches"]),
        "clocks": mixed["clocks"],
        "error_vs_fp64_oracle": err,
        "time_to_energy_tol": tte,
        "setup": setup,
    }
    if ws == 1 and not args.no_cpu_baseline:  # a reported baseline at N = 1 only
        line["cpu_baseline"] = cpu_baseline()
    if ws == 1 and not args.no_configs and args.only is None and args.n == N_SIDE:
        line["configs"] = side_configs(args, local)
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
