#!/usr/bin/env python
"""Benchmark of the per-step residual-and-implicit-update path on B200.

    python bench.py [--gpus N --steps K --warmup W] [--impl b200|reference]
                    [--config reacting_step|flat_plate|sod|reactors|adjoint|cea] [--scale S]

Metric: Mcell-iter/s (cells x inner iterations per second; for the explicit
Euler configuration one step is one iteration), mixed (FP32 reconstruction,
fluxes and sweeps) and plain FP64.  `value` is the mixed path with the state
resident in HBM; `fp64_value` the plain path; `e2e` the same metric through the
C ABI with host buffers copied in and the result copied out every step.

--config reactors measures the batched 0-D reactors instead: reactors/s for
one batch of 8192 H2/air reactors integrated to 2 ms (a step is one batch).
--config cea measures the CEA equilibrium solve: Mcell/s over 2^22 cells, each
step a warm-started re-solve of every cell.

One JSON line is printed by rank 0.  Under torchrun (N > 1) the flow
configurations are block-sharded over the ranks (strong scaling: the same
workload; each block is cut along i into ceil(N/2) pieces for the four-block
reacting step, N pieces for a single-block case, and the pieces are spread
evenly by cell count): halo cells travel by NCCL all-gather, dt, the inner
residual, omega and the status by NCCL all-reduce, all on the library's
stream.  --sharded takes that path also at N = 1.  The reactors are
independent units: each rank integrates its own batch (weak scaling, no data
exchange).  Times are the maximum over ranks.
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from shared_cfd_b200 import abi, cases  # noqa: E402


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def make_case(config, scale, precision):
    if config == "reacting_step":
        return cases.reacting_step(scale=scale, precision=precision)
    if config == "flat_plate":
        return cases.flat_plate(int(round(256 * scale)), int(round(128 * scale)), precision=precision)
    return cases.sod(int(round(400 * scale)), 4, precision=precision)


def shard_pieces(config, world):
    """Pieces per block along i for a run over `world` ranks."""
    if world <= 1:
        return 1
    return (world + 1) // 2 if config == "reacting_step" else world


def unit_of(config):
    return "Mcell-step/s" if config == "sod" else "Mcell-iter/s"


def unit_of_case(case):
    return "Mcell-step/s" if case.desc.scheme == abi.SCHEME_EULER else "Mcell-iter/s"


def iters_per_step(case):
    return max(1, case.desc.num_internal_loop - 1) if case.desc.scheme == abi.SCHEME_NR else 1


METRIC = {
    "reacting_step": "Mcell-iter/s of the reacting-step NR dual-time step (cells x inner iterations per second)",
    "flat_plate": "Mcell-iter/s of the flat-plate LU-SGS step (cells x iterations per second)",
    "sod": "Mcell-step/s of the Sod explicit step (cells x steps per second)",
}


def workload_name(config, scale):
    return {"reacting_step": "axisymmetric reacting backward-facing step, 4 blocks 2x512^2+2x512x256, "
                             "9 species / 19 seeded reactions, NR dual time dt=1e-7 s, 20 inner iterations",
            "flat_plate": "supersonic laminar flat plate 256x128, N2 Sutherland Pr=0.72, LU-SGS local dt",
            "sod": "Sod shock tube 400x4, MUSCL+SLAU, explicit Euler CFL 0.5"}[config] + \
        ("" if scale == 1.0 else " (scale %g)" % scale)


# DRAM bytes (read + write) per interior cell and launch, from ncu captures of the
# reacting step at scale 0.5 (196 608 cells; ncu flushes the caches before each
# launch, so reads are cold, and writes still in L2 at a launch's end are not
# counted); commands in profiles/traffic_reacting_step_196k.md, which also says which
# build each figure was captured on (the sweeps and the FP64 residual on this one).
# None of these kernels reuses data across launches, so the traffic of a launch grows
# with the cell count and is scaled to the workload by cells.  K_UPDATE averages its
# two launches per inner iteration (k_omega and k_unpack).
NCU_DRAM_BYTES_PER_CELL = {
    ("reacting_step", False): {abi.K_THERMO: 159.3, abi.K_RESIDUAL: 656.0, abi.K_PACK: 542.1,
                               abi.K_SWEEP_FWD: 447.3, abi.K_SWEEP_BWD: 437.7, abi.K_UPDATE: 197.0},
    ("reacting_step", True): {abi.K_THERMO: 159.3, abi.K_RESIDUAL: 553.9, abi.K_PACK: 404.7,
                              abi.K_SWEEP_FWD: 216.2, abi.K_SWEEP_BWD: 216.2, abi.K_UPDATE: 143.2},
}
NCU_TRAFFIC_NOTE = "ncu dram__bytes_read+write per cell at scale 0.5 (cold cache), scaled by cells"


def traffic_per_launch(config, mixed, kind, ncells):
    t = NCU_DRAM_BYTES_PER_CELL.get((config, mixed), {}).get(kind)
    return None if t is None else t * ncells


def algo_bytes(kind, case, mixed):
    nY, D, W = case.nY, case.D, case.W
    nr = case.desc.scheme == abi.SCHEME_NR
    wb = 4 if mixed else 8
    if kind == abi.K_THERMO:
        return 8 * ((D + 2) + W + 2 * nY)
    if kind == abi.K_RESIDUAL:
        geo = 28 if case.desc.viscous else 14
        return wb * (W + nY) + 8 * ((3 * D if nr else 2 * D) + geo + D + 3)
    if kind in (abi.K_SWEEP_FWD, abi.K_SWEEP_BWD):
        return 8 * (D + 1 + 4 + 2 * nY + 2 + 4 + 2 + 1 + D)
    if kind == abi.K_UPDATE:
        # NR: k_omega (Dq of the species and energy, q of the species) and k_unpack
        # (q += omega Dq), averaged over the two launches
        return (8 * (2 * nY + 1) + 8 * 3 * D) // 2 if nr else 8 * 3 * D
    if kind == abi.K_BC:
        return 0
    if kind == abi.K_CHEM:
        return 8 * (2 * nY + 3)
    return 0


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.f = None
        self.skip = 0

    def __enter__(self):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
            return self
        # the first sample takes a moment: start timing only once it is in
        t0 = time.time()
        while time.time() - t0 < 5.0 and os.path.getsize(self.f.name) == 0 and self.proc.poll() is None:
            time.sleep(0.02)
        with open(self.f.name) as f:
            self.skip = len([r for r in f.read().splitlines() if r.strip()])
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.f.flush()

    def summary(self):
        try:
            with open(self.f.name) as f:
                rows = [r.split(",") for r in f.read().strip().splitlines() if r.strip()]
            os.unlink(self.f.name)
            # samples taken before the timed region began are dropped (kept
            # when nothing else arrived, so that a short region still reports)
            if len(rows) > self.skip:
                rows = rows[self.skip:]
        except OSError:
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[0]))
                mx = float(r[1])
                for k, nm in enumerate(names):
                    if r[4 + k].strip().lower().startswith("active"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def time_resident(solver, steps, warmup, torch, dev, sampler_dev, barrier):
    """Device time of `steps` steps with the state resident (CUDA events on the
    library's stream), after `warmup` untimed steps."""
    stream = torch.cuda.ExternalStream(solver.stream(), device=dev)
    if warmup:
        solver.run(1, warmup)
    barrier()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(sampler_dev) as cs:
        e0.record(stream)
        st = solver.run(1 + warmup, steps)
        e1.record(stream)
        torch.cuda.synchronize(dev)
    barrier()
    return e0.elapsed_time(e1), st, solver.launch_count(), cs.summary()


def kernel_profile(solver, steps, case, mixed, ncells=None):
    ncells = case.ncells if ncells is None else ncells
    lib = solver.lib
    lib.profile(solver.ctx, 1)
    solver.run(100, steps)
    out = {}
    for k in range(abi.K_COUNT):
        ms = C.c_double()
        n = C.c_int64()
        name = C.create_string_buffer(32)
        lib.kernel_stats(solver.ctx, k, C.byref(ms), C.byref(n), name, 32)
        if n.value:
            out[name.value.decode()] = {"kind": k, "total_ms": ms.value, "launches": n.value,
                                        "avg_ms": ms.value / n.value,
                                        "bytes_per_launch": algo_bytes(k, case, mixed) * ncells}
    lib.profile(solver.ctx, 0)
    return out


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    except (OSError, ValueError):
        return 6650.0, "fallback"


def cpu_reference(config, scale, steps, cores, threads=None):
    """The CPU restatement of the reference (OpenMP on the host cores; `threads`
    caps the OpenMP team of this and later runs)."""
    from shared_cfd_b200.solver import Solver
    so = os.path.join(ROOT, "oracle", "_build", "liborc.so")
    if not os.path.exists(so):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    os.environ["OMP_NUM_THREADS"] = str(cores)
    orc = abi.Bound(C.CDLL(so), "orc_")
    if threads is not None:
        import ctypes.util
        C.CDLL(ctypes.util.find_library("gomp") or "libgomp.so.1").omp_set_num_threads(threads)
    case = make_case(config, scale, abi.PREC_FP64)
    s = Solver(case, lib=orc)
    s.upload()
    s.prepare(1)
    t0 = time.perf_counter()
    st = s.run(1, steps, check=False)
    dt = time.perf_counter() - t0
    q = s.download()[0]
    s.close()
    units = case.ncells * iters_per_step(case) * steps
    return units / dt / 1e6, dt, case, q, st.status


def l2_note(case):
    """Working set of one inner iteration against the 126 MB L2 (no flush is done)."""
    D, W, nY = case.D, case.W, case.nY
    # FP64 per cell: q, qp, qpp, Dq (D each), w (W), vhi, DHi (nY each), geometry (~16),
    # dt; FP32 copies of w and vhi; one strip record (about 5 D values)
    per_cell = 8 * (4 * D + W + 2 * nY + 17) + 4 * (W + nY) + 4 * (5 * D)
    mb = per_cell * case.ncells / 1e6
    if mb > 126:
        return "working set ~%.0f MB per inner iteration > 126 MB L2 (no flush)" % mb
    return "working set ~%.0f MB fits the 126 MB L2" % mb


# ---------------------------------------------------------------------------
# batched 0-D reactors (scfd_reactors_*)
# ---------------------------------------------------------------------------
REACTOR_N = 8192
REACTOR_T_END = 2e-3
REACTOR_DT_CALL = 1e-6


def reactor_flops_per_eval(ns, nr):
    """Algorithmic flops of one Fex_var evaluation (an estimate, the unit of the
    reactors' FP64 roofline): NASA-7 thermo, 3 x 7 multiply-adds per species and
    the T sums (~45 flops per species); per reaction the Arrhenius exponent,
    concentration products and two exponentials counted at ~20 flops each (~60)."""
    return 45 * ns + 60 * nr


def reactor_workload():
    return ("%d constant-volume H2/air 0-D reactors (T0 900-1600 K, p 1-20 atm, phi 0.3-3), reacting-step "
            "mechanism (9 species, 19 seeded reactions), CHEMEQ2 calls every %g s to %g s" %
            (REACTOR_N, REACTOR_DT_CALL, REACTOR_T_END))


def cpu_reactors(cores, n=None):
    n = REACTOR_N if n is None else n
    from shared_cfd_b200.reactors import Reactors
    so = os.path.join(ROOT, "oracle", "_build", "liborc.so")
    if not os.path.exists(so):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    os.environ["OMP_NUM_THREADS"] = str(cores)
    orc = abi.Bound(C.CDLL(so), "orc_")
    _, ch, T0, v, _ = cases.reactor_batch(n)
    with Reactors(ch, n, lib=orc) as r:
        t0 = time.perf_counter()
        out = r.run(T0, v, REACTOR_T_END, dt_call=REACTOR_DT_CALL)
        dt = time.perf_counter() - t0
    return n / dt, dt, out


# ---------------------------------------------------------------------------
# discrete adjoint of the explicit ideal-gas step (scfd_adjoint_run)
# ---------------------------------------------------------------------------
ADJ_N, ADJ_STEPS, ADJ_WINDOW, ADJ_SNAPSHOTS = 256, 300, (200, 299), 16


def adjoint_workload():
    return ("gradient of the pressure force on a slip wall (steps %d-%d) with respect to the inflow state: "
            "2 ideal-gas blocks 256x256 + 512x256 (196 608 cells), MUSCL + SLAU, explicit Euler, %d steps, "
            "binomial checkpointing with %d stored states" % (ADJ_WINDOW[0], ADJ_WINDOW[1], ADJ_STEPS, ADJ_SNAPSHOTS))


def run_adjoint(args, rank, cores):
    """One JSON line: primal and adjoint device time of the same run; value =
    cell-steps per second of the gradient computation."""
    unit = "Mcell-step/s"
    case = cases.adjoint_channel(n=ADJ_N)
    units = case.ncells * ADJ_STEPS / 1e6
    if args.impl == "reference":
        if rank != 0:
            return 0
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no adjoint (and no tangent-linear "
                          "model); only the primal objective is restated on the CPU"}), flush=True)
        return 0
    if rank != 0:
        return 0
    import torch
    from shared_cfd_b200 import build
    from shared_cfd_b200.adjoint import adjoint_run
    from shared_cfd_b200.solver import Solver
    build.build()
    s = Solver(case)
    s.upload()
    stream = torch.cuda.ExternalStream(s.stream(), device=0)
    for _ in range(max(1, args.warmup)):
        adjoint_run(s, 4, 2, (1, 3), 0, snapshots=2)
        s.upload()
        s.run(1, 3)
        s.upload()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    prim, adj = [], []
    with ClockSampler(0) as cs:
        for _ in range(max(1, args.steps)):
            torch.cuda.synchronize()
            e0.record(stream)
            st = s.run(1, ADJ_STEPS)
            e1.record(stream)
            torch.cuda.synchronize()
            prim.append(e0.elapsed_time(e1))
            s.upload()
            t0 = time.perf_counter()
            J, grad, counts = adjoint_run(s, ADJ_STEPS, 2, ADJ_WINDOW, 0, snapshots=ADJ_SNAPSHOTS)
            adj.append(1e3 * (time.perf_counter() - t0))
    ms_p, ms_a = min(prim), min(adj)
    q = s.download()[0]
    s.close()
    line = {
        "metric": "Mcell-step/s of the adjoint gradient (FP64)", "value": units / (ms_a * 1e-3), "unit": unit,
        "n_gpus": 1, "steps": max(1, args.steps), "warmup": args.warmup, "ms_per_step": ms_a,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": adjoint_workload(), "cells": case.ncells, "steps": ADJ_STEPS},
        "adjoint_over_primal": ms_a / ms_p, "primal_ms": ms_p, "adjoint_ms": ms_a,
        "forward_steps": counts[0], "reverse_steps": counts[1], "J": J,
        "grad_inflow": {"rho": grad[0], "u": grad[1], "v": grad[2], "p": grad[3]},
        "primal_status": st.status, "state_finite": bool(np.isfinite(q).all()),
        "e2e": None, "cpu_baseline": None,
        "clocks": cs.summary(),
        "note": "primal = the same %d steps through scfd_run (CUDA graph); the adjoint time is host wall time of "
                "scfd_adjoint_run (its forward recomputation, reverse steps and state copies)" % ADJ_STEPS,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_reactors(args, rank, cores):
    """One JSON line for the 0-D reactor batch (rank 0 only; the batch does not
    shard across ranks in this benchmark)."""
    unit = "reactors/s"
    if args.impl == "reference":
        if rank != 0:
            return 0
        steps = max(1, args.steps)
        t = 0.0
        for _ in range(steps):
            _, dt, _ = cpu_reactors(cores)
            t += dt
        val = REACTOR_N * steps / t
        print(json.dumps({
            "impl": "reference", "metric": "reactors/s (0-D, FP64)", "value": val, "unit": unit,
            "n_gpus": args.gpus, "steps": steps, "warmup": 0, "ms_per_step": 1e3 * t / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": {"workload": reactor_workload()},
            "cpu_baseline": {"value": val, "unit": unit, "cores": cores, "kind": "port",
                             "sample": "%d batch(es) of %d reactors on %d OpenMP threads (C++ FP64 restatement)"
                                       % (steps, REACTOR_N, cores)},
            "e2e": {"value": val, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)
        return 0
    if rank != 0:
        return 0
    import torch
    from shared_cfd_b200 import build
    from shared_cfd_b200.reactors import Reactors
    build.build()
    m, ch, T0, v, _ = cases.reactor_batch(REACTOR_N)
    r = Reactors(ch, REACTOR_N)
    d = r.desc(REACTOR_N, REACTOR_T_END, dt_call=REACTOR_DT_CALL)
    stream = torch.cuda.ExternalStream(r.stream(), device=0)
    r.upload(T0, v)
    for _ in range(max(1, args.warmup)):
        r.launch(d)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as cs:
        e0.record(stream)
        for _ in range(args.steps):
            r.launch(d)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    out = r.download(REACTOR_N)
    launches = r.launch_count() * args.steps
    value = REACTOR_N / (ms * 1e-3)
    # end to end: host arrays in, results out, every batch
    t0 = time.perf_counter()
    for _ in range(args.steps):
        r.run(T0, v, REACTOR_T_END, dt_call=REACTOR_DT_CALL)
    e2e_s = (time.perf_counter() - t0) / args.steps
    # one kernel launch per reactor, on a bounded sample (serial by construction)
    ns_pl = 64
    t0 = time.perf_counter()
    r.run(T0[:ns_pl], v[:ns_pl], REACTOR_T_END, mode=abi.REACTOR_PER_LAUNCH, dt_call=REACTOR_DT_CALL)
    pl_s = time.perf_counter() - t0
    r.close()
    evals = int(out["evals"].sum())
    flops = evals * reactor_flops_per_eval(ch.ns, ch.nr)
    ach = flops / (ms * 1e-3) / 1e9
    line = {
        "metric": "reactors/s (0-D, FP64)", "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": reactor_workload(), "reactors": REACTOR_N, "mode": "persistent work queue, CUDA graph",
                   "l2": "state of all reactors (~1 MB) is L2-resident; the kernel is latency-bound"},
        "e2e": {"value": REACTOR_N / e2e_s, "unit": unit,
                "h2d_bytes_per_step": int(T0.nbytes + v.nbytes),
                "d2h_bytes_per_step": int(T0.nbytes * 3 + v.nbytes + out["flags"].nbytes)},
        "gpu_launches": launches, "clocks": cs.summary(),
        "per_launch": {"value": ns_pl / pl_s, "unit": unit, "sample": "first %d reactors, one launch each" % ns_pl},
        "roofline": {"bound": "fp64", "achieved": ach, "peak": 40000.0, "unit": "GFLOP/s", "frac": ach / 40000.0,
                     "peak_source": "nominal B200 FP64 (not measured)", "traffic": None,
                     "flops_per_eval": reactor_flops_per_eval(ch.ns, ch.nr), "evals_per_batch": evals},
        "reactors": {"ignited": int(((out["flags"] & abi.REACTOR_IGNITED) > 0).sum()),
                     "fell_back": int(((out["flags"] & abi.REACTOR_FELL_BACK) > 0).sum()),
                     "failed": int(((out["flags"] & abi.REACTOR_FAILED) > 0).sum()),
                     "evals_max": int(out["evals"].max()), "status": int(out["status"])},
    }
    if not args.no_cpu_baseline:
        v_cpu, dt, ref = cpu_reactors(cores)
        ign = (ref["flags"] & abi.REACTOR_IGNITED) > 0
        line["cpu_baseline"] = {"value": v_cpu, "unit": unit, "cores": cores, "kind": "port",
                                "sample": "the full batch (%.1f s) on %d OpenMP threads, C++ FP64 restatement"
                                          % (dt, cores)}
        line["accuracy_vs_cpu"] = {
            "flags_differ": int((ref["flags"] != out["flags"]).sum()),
            "t_ign_max_rel": float(np.max(np.abs(out["t_ign"][ign] - ref["t_ign"][ign]) / ref["t_ign"][ign]))
            if ign.any() else None,
            "T_end_max_rel": float(np.max(np.abs(out["T_end"] - ref["T_end"]) / ref["T_end"])),
            "T_end_median_rel": float(np.median(np.abs(out["T_end"] - ref["T_end"]) / ref["T_end"]))}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# CEA chemical equilibrium (scfd_cea_solve)
# ---------------------------------------------------------------------------
CEA_N = 1 << 22
CEA_DE = 0.01


def cea_workload():
    return ("%d cells of CEA chemical equilibrium at fixed density, energy and fuel / oxidizer mass fractions: "
            "H2 against air over 9 H/O/N species (3 elements, NASA-9 data); seeded states (Y_fuel = u^3, "
            "rho 0.2-2 kg/m^3, e = mixed-stream e + 0-3 MJ/kg); each step re-solves every cell from the previous "
            "step's T and n with e alternately raised and lowered by %g of |e| (the warm start of the flow "
            "model's saved n)" % (CEA_N, CEA_DE))


def cea_states(info):
    from shared_cfd_b200 import cea
    rho, Y, e, T = cea.random_states(info, CEA_N, seed=21)
    return rho, Y, e, e + CEA_DE * np.abs(e), T


def cpu_cea(cores, seconds=10.0):
    """The CPU restatement on the benchmark workload: one cold solve
    (untimed), then warm steps until `seconds` have passed (at least 2)."""
    from shared_cfd_b200 import cea
    so = os.path.join(ROOT, "oracle", "_build", "liborc.so")
    if not os.path.exists(so):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    os.environ["OMP_NUM_THREADS"] = str(cores)
    orc = abi.Bound(C.CDLL(so), "orc_")
    with cea.Cea(cea.h2_air_data(), lib=orc) as m:
        rho, Y, e0, e1, T = cea_states(m.info())
        n = m.initial_n(CEA_N)
        Tp = np.empty(CEA_N)
        np.copyto(Tp, T)
        z = np.zeros(CEA_N)
        zs = np.zeros((m.ns, CEA_N))
        zz = np.zeros((m.ns, CEA_N))
        d2 = np.zeros((2, CEA_N))
        it = np.zeros(CEA_N, dtype=np.int32)
        z1, z2 = np.zeros(CEA_N), np.zeros(CEA_N)

        def step(e):
            m.solve_ptr(CEA_N, rho.ctypes.data, Y.ctypes.data, e.ctypes.data, Tp.ctypes.data, n.ctypes.data,
                        z.ctypes.data, z1.ctypes.data, z2.ctypes.data, zs.ctypes.data, zz.ctypes.data,
                        d2.ctypes.data, it.ctypes.data, None)
        step(e0)
        k, t0 = 0, time.perf_counter()
        while k < 2 or time.perf_counter() - t0 < seconds:
            step(e1 if k % 2 == 0 else e0)
            k += 1
        dt = time.perf_counter() - t0
        return CEA_N * k / dt / 1e6, dt, k


def run_cea(args, rank, cores):
    """One JSON line for the CEA equilibrium batch (rank 0 only; the cells are
    independent and the benchmark does not shard them)."""
    unit = "Mcell/s"
    metric = "Mcell/s of CEA equilibrium solves (FP64)"
    if args.impl == "reference":
        if rank != 0:
            return 0
        val, dt, k = cpu_cea(cores)
        print(json.dumps({
            "impl": "reference", "metric": metric, "value": val, "unit": unit, "n_gpus": args.gpus, "steps": k,
            "warmup": 1, "ms_per_step": 1e3 * dt / k, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "config": {"workload": cea_workload()},
            "cpu_baseline": {"value": val, "unit": unit, "cores": cores, "kind": "port",
                             "sample": "%d warm steps of the full workload (%.1f s) on %d OpenMP threads, C++ FP64 "
                                       "restatement of cea" % (k, dt, cores)},
            "e2e": {"value": val, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)
        return 0
    if rank != 0:
        return 0
    import torch
    from shared_cfd_b200 import build, cea
    build.build()
    g = cea.Cea(cea.h2_air_data())
    info = g.info()
    ns = g.ns
    rho, Y, e0, e1, T = cea_states(info)
    dev = torch.device("cuda", 0)

    def t(a):
        return torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    d = {"rho": t(rho), "Y": t(Y), "e0": t(e0), "e1": t(e1), "T": t(T), "n": t(np.full((ns, CEA_N), info.n_init))}
    outs = [torch.empty(CEA_N, dtype=torch.float64, device=dev) for _ in range(3)] + \
        [torch.empty((ns, CEA_N), dtype=torch.float64, device=dev) for _ in range(2)] + \
        [torch.empty((2, CEA_N), dtype=torch.float64, device=dev)]
    it = torch.empty(CEA_N, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def solve(e):
        g.solve_device(d["rho"], d["Y"], e, d["T"], d["n"], *outs, iters=it, stream=stream)

    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    # cold start from the initial n_save: one launch, its own sub-measure
    torch.cuda.synchronize(dev)
    ev[0].record(stream)
    solve(d["e0"])
    ev[1].record(stream)
    torch.cuda.synchronize(dev)
    cold_ms = ev[0].elapsed_time(ev[1])
    cold_it = float(it.float().mean())
    code, nc, ng = g.status()
    if code or ng:
        raise RuntimeError("cea status %d (%d singular)" % (code, ng))
    k = 0
    for _ in range(max(3, args.warmup)):
        solve(d["e1"] if k % 2 == 0 else d["e0"])
        k += 1
    torch.cuda.synchronize(dev)
    with ClockSampler(0) as cs:
        ev[0].record(stream)
        for _ in range(args.steps):
            solve(d["e1"] if k % 2 == 0 else d["e0"])
            k += 1
        ev[1].record(stream)
        torch.cuda.synchronize(dev)
    ms = ev[0].elapsed_time(ev[1]) / args.steps
    warm_it = float(it.float().mean())
    code, nc, ng = g.status()
    if code or ng:
        raise RuntimeError("cea status %d (%d singular)" % (code, ng))
    value = CEA_N / (ms * 1e-3) / 1e6
    # end to end through the same call with host buffers: the step's inputs
    # (rho, Y, e, T, n) copied in from pinned memory, every output copied back
    hp = {k_: torch.from_numpy(np.ascontiguousarray(v)).pin_memory() for k_, v in
          (("rho", rho), ("Y", Y), ("e0", e0), ("e1", e1))}
    hT = d["T"].cpu().pin_memory()
    hn = d["n"].cpu().pin_memory()
    hout = [torch.empty(o.shape, dtype=o.dtype).pin_memory() for o in outs]
    dd = {k_: torch.empty_like(d[k_]) for k_ in ("rho", "Y", "T", "n")}
    de = torch.empty_like(d["e0"])

    def e2e_step(e_host):
        dd["rho"].copy_(hp["rho"], non_blocking=True)
        dd["Y"].copy_(hp["Y"], non_blocking=True)
        de.copy_(e_host, non_blocking=True)
        dd["T"].copy_(hT, non_blocking=True)
        dd["n"].copy_(hn, non_blocking=True)
        g.solve_device(dd["rho"], dd["Y"], de, dd["T"], dd["n"], *outs, stream=stream)
        hT.copy_(dd["T"], non_blocking=True)
        hn.copy_(dd["n"], non_blocking=True)
        for h, o in zip(hout, outs):
            h.copy_(o, non_blocking=True)
        torch.cuda.synchronize(dev)
    for _ in range(2):
        e2e_step(hp["e1"] if k % 2 == 0 else hp["e0"])
        k += 1
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step(hp["e1"] if k % 2 == 0 else hp["e0"])
        k += 1
    e2e_s = (time.perf_counter() - t0) / args.steps
    g.close()
    h2d = 8 * CEA_N * (1 + 2 + 1 + 1 + ns)
    d2h = 8 * CEA_N * (1 + ns + 3 + 2 * ns + 2)
    peak, src = measured_peaks()
    bpl = 8 * CEA_N * ((1 + 2 + 1 + 1 + ns) + (1 + ns + 3 + 2 * ns + 2))
    ach = bpl / (ms * 1e-3) / 1e9
    line = {
        "metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": cea_workload(), "cells": CEA_N,
                   "l2": "inputs and outputs (%d MB per step) are larger than L2" % (bpl // 10**6)},
        "newton_iterations_mean": warm_it,
        "cold_start": {"value": CEA_N / (cold_ms * 1e-3) / 1e6, "unit": unit, "newton_iterations_mean": cold_it,
                       "note": "one launch from the initial n_save (sum(no + nf) / ns in every cell)"},
        "e2e": {"value": CEA_N / e2e_s / 1e6, "unit": unit, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": args.steps, "clocks": cs.summary(),
        "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                     "peak_source": src, "traffic": None, "bytes_per_cell": bpl // CEA_N,
                     "note": "the kernel is FP64 latency-bound (a Newton iteration of exp / log per species per "
                             "cell); HBM carries only its inputs and outputs"},
    }
    if not args.no_cpu_baseline:
        v_cpu, dt, kc = cpu_cea(cores)
        line["cpu_baseline"] = {"value": v_cpu, "unit": unit, "cores": cores, "kind": "port",
                                "sample": "%d warm steps of the full workload (%.1f s) on %d OpenMP threads, C++ FP64 "
                                          "restatement of cea" % (kc, dt, cores)}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="reacting_step",
                    choices=["reacting_step", "flat_plate", "sod", "reactors", "adjoint", "cea"])
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--cpu-steps", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sharded", action="store_true", help="block-sharded path also at N = 1 (needs torchrun)")
    ap.add_argument("--cea-cells", type=int, default=0, help="cells of --config cea (default 2^22)")
    ap.add_argument("--reactors-n", type=int, default=0, help="reactors of --config reactors (default 8192)")
    ap.add_argument("--reactors-t-end", type=float, default=0.0, help="end time of --config reactors (default 2e-3 s)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    cores = os.cpu_count() or 1

    if args.config == "reactors":
        global REACTOR_N, REACTOR_T_END
        if args.reactors_n > 0:
            REACTOR_N = args.reactors_n
        if args.reactors_t_end > 0.0:
            REACTOR_T_END = args.reactors_t_end
        return run_reactors(args, rank, cores)
    if args.config == "adjoint":
        return run_adjoint(args, rank, cores)
    if args.config == "cea":
        if args.cea_cells > 0:
            global CEA_N
            CEA_N = args.cea_cells
        return run_cea(args, rank, cores)

    if args.impl == "reference":
        if rank != 0:
            return 0
        steps = max(1, args.steps)
        val, dt, case, _, _ = cpu_reference(args.config, args.scale, steps, cores)
        unit = unit_of(args.config)
        line = {"impl": "reference", "metric": METRIC[args.config], "value": val, "unit": unit,
                "n_gpus": args.gpus, "steps": steps, "warmup": 0, "ms_per_step": 1e3 * dt / steps,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded)",
                "config": {"workload": workload_name(args.config, args.scale), "cells": case.ncells,
                           "inner_iterations": iters_per_step(case), "controls": controls_note(case)},
                "cpu_baseline": {"value": val, "unit": unit, "cores": cores, "kind": "port",
                                 "sample": "%d physical step(s) of the full workload on %d OpenMP threads "
                                           "(C++ FP64 restatement of the reference)" % (steps, cores)},
                "e2e": {"value": val, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    import torch
    dev = local if torch.cuda.device_count() > 1 else 0
    torch.cuda.set_device(dev)
    dist = None
    sharded = world > 1 or args.sharded
    if sharded:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", dev))

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    from shared_cfd_b200 import build
    from shared_cfd_b200.sharded import ShardedSolver, partition_planes
    from shared_cfd_b200.solver import Solver
    if rank == 0:
        build.build()
    barrier()

    unit = unit_of(args.config)
    res = {}
    solvers = {}
    q_after = {}
    pieces = shard_pieces(args.config, world)
    for prec, tag in ((abi.PREC_FP64, "fp64"), (abi.PREC_MIXED, "mixed")):
        case = make_case(args.config, args.scale, prec)
        if sharded:
            case = cases.split_planes_i(case, pieces)
            owner = partition_planes([a * b for a, b in zip(case.ni, case.nj)], world)
            s = ShardedSolver(case, owner)
        else:
            s = Solver(case)
        s.upload()
        s.prepare(1)
        ms, st, nl, clk = time_resident(s, args.steps, args.warmup, torch, dev, dev, barrier)
        ms = max_over_ranks(ms)
        # the state after the warm-up and timed steps, for the mixed-vs-FP64 error
        q_after[tag] = s.gather()[0] if sharded else s.download()[0]
        # strong scaling under sharding: the ranks share one workload
        units = case.ncells * iters_per_step(case) * args.steps * (1 if sharded else world)
        om, rr = s.inner_log() if case.desc.scheme == abi.SCHEME_NR else (np.zeros(0), np.zeros(0))
        res[tag] = {"ms": ms, "value": units / (ms * 1e-3) / 1e6, "launches": nl, "clocks": clk,
                    "autotune": s.tuning(), "status": st.status, "res_warn": st.res_warn, "omega": st.omega,
                    "chem_attempts": st.chem_attempts, "chem_fallback": st.chem_fallback_cells,
                    "inner_omega": [float(x) for x in om], "inner_res_ratio": [float(x / rr[0]) for x in rr]}
        solvers[tag] = (s, case)
        log("%s: %.2f ms/step  %.1f %s  status %d" % (tag, ms / args.steps, res[tag]["value"], unit, st.status))

    peak, peak_kind = measured_peaks()
    prof, roof = {}, {}
    for tag in ("fp64", "mixed"):
        s_k, case_k = solvers[tag]
        cells_here = s_k.owned_cells if sharded else case_k.ncells
        prof[tag] = kernel_profile(s_k, args.steps, case_k, tag == "mixed", cells_here)
        roof[tag] = roofline_of(prof[tag], args.config, tag == "mixed", cells_here, peak, peak_kind)

    # end to end through the C ABI with host buffers, both precisions
    e2e = {tag: e2e_run(*solvers[tag], args.steps, sharded, world, barrier, max_over_ranks, torch, dev)
           for tag in ("fp64", "mixed")}

    # the CPU restatement on the same workload: the timed baseline, and the
    # oracle state both GPU paths are compared with after the same steps
    cpu, acc = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            v, dt, _, q_orc, orc_status = cpu_reference(args.config, args.scale, args.cpu_steps, cores)
            cpu = {"value": v, "unit": unit, "cores": cores, "kind": "port",
                   "sample": "%d physical step(s) of the full workload (%.1f s) on %d OpenMP threads, "
                             "C++ FP64 restatement" % (args.cpu_steps, dt, cores)}
            # one core, on a quarter-resolution sample of the same case (1/16 of the cells)
            v1, dt1, c1, _, _ = cpu_reference(args.config, args.scale * 0.25, 1, cores, threads=1)
            cpu["single_core"] = {"value": v1, "unit": unit, "cores": 1,
                                  "sample": "1 physical step of the workload at quarter resolution per "
                                            "direction (%d cells, %.1f s) on 1 thread" % (c1.ncells, dt1)}
            acc = accuracy_vs_oracle(args, q_orc, orc_status)
        except Exception as e:  # noqa: BLE001
            cpu = {"value": None, "unit": unit, "cores": cores, "kind": "port", "sample": "failed: %s" % e}

    # the mixed path against the FP64 path after the same warm-up + timed steps
    # from the same initial state
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import rel_l2
    l2_mixed_fp64 = rel_l2(solvers["fp64"][1], q_after["mixed"], q_after["fp64"])

    if rank == 0:
        d, m = res["fp64"], res["mixed"]
        case = solvers["fp64"][1]
        line = {
            "metric": METRIC[args.config],
            "value": d["value"], "unit": unit, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": d["ms"] / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": workload_name(args.config, args.scale), "cells": case.ncells,
                       "inner_iterations": iters_per_step(case),
                       "parallelism": ("%d GPU(s), block-sharded: %d planes (blocks cut along i into %d), "
                                       "NCCL all-gather of halo cells and all-reduce of dt/res/omega/status"
                                       % (world, len(case.planes), pieces)) if sharded else "1 GPU",
                       "l2": l2_note(case), "controls": controls_note(case)},
            "e2e": e2e["fp64"], "gpu_launches": d["launches"], "clocks": d["clocks"],
            "roofline": roof["fp64"], "cpu_baseline": cpu,
            "accuracy": acc,
            "status": {"code": d["status"], "res_warn": d["res_warn"], "omega": d["omega"],
                       "chem_attempts": d["chem_attempts"], "chem_fallback_cells": d["chem_fallback"],
                       "last_step_inner_omega": d["inner_omega"], "last_step_inner_res_ratio": d["inner_res_ratio"]},
            "mixed": {"value": m["value"], "unit": unit, "ms_per_step": m["ms"] / args.steps,
                      "over_fp64": m["value"] / d["value"], "e2e": e2e["mixed"], "gpu_launches": m["launches"],
                      "clocks": m["clocks"], "roofline": roof["mixed"],
                      "l2_vs_fp64_gpu": {"value": l2_mixed_fp64, "steps": args.warmup + args.steps},
                      "dtype": "f32 reconstruction, fluxes and sweeps; f64 thermo, chemistry, sums, updates",
                      "status": {"code": m["status"], "omega": m["omega"],
                                 "last_step_inner_omega": m["inner_omega"]}},
            "autotune": {"fp64": d["autotune"], "mixed": m["autotune"]},
            "kernels_fp64": {k: {kk: v[kk] for kk in ("avg_ms", "launches", "total_ms", "gbs") if kk in v}
                             for k, v in prof["fp64"].items()},
            "kernels_mixed": {k: {kk: v[kk] for kk in ("avg_ms", "launches", "total_ms", "gbs") if kk in v}
                              for k, v in prof["mixed"].items()},
        }
        print(json.dumps(line), flush=True)
    for s, _ in solvers.values():
        s.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def roofline_of(prof, config, mixed, cells_here, peak, peak_kind):
    """Roofline of the dominant HBM-touching kernel of one precision's profile,
    and the same for the face-flux kernel."""
    hbm = {k: v for k, v in prof.items() if v["bytes_per_launch"] > 0 and v["kind"] != abi.K_CHEM}
    top = max(prof.items(), key=lambda kv: kv[1]["total_ms"])
    dom = max(hbm.items(), key=lambda kv: kv[1]["total_ms"]) if hbm else top
    ach = dom[1]["bytes_per_launch"] / (dom[1]["avg_ms"] * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": dom[0], "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": ach / peak, "peak_source": peak_kind,
                "traffic": traffic_per_launch(config, mixed, dom[1]["kind"], cells_here),
                "traffic_source": NCU_TRAFFIC_NOTE,
                "algorithmic_bytes_per_launch": dom[1]["bytes_per_launch"],
                "avg_launch_ms": dom[1]["avg_ms"], "top_kernel_by_time": top[0]}
    if "residual" in prof:
        r = prof["residual"]
        ach_r = r["bytes_per_launch"] / (r["avg_ms"] * 1e-3) / 1e9
        roofline["flux_kernel"] = {"kernel": "residual", "achieved": ach_r, "frac": ach_r / peak,
                                   "traffic": traffic_per_launch(config, mixed, abi.K_RESIDUAL, cells_here),
                                   "avg_launch_ms": r["avg_ms"]}
    for v in prof.values():
        if v["bytes_per_launch"]:
            v["gbs"] = v["bytes_per_launch"] / (v["avg_ms"] * 1e-3) / 1e9
    return roofline


def e2e_run(s_e, case_e, steps, sharded, world, barrier, max_over_ranks, torch, dev):
    """The metric through scfd_upload / scfd_step / scfd_download with host
    buffers every step (the reference-layout arrays cross PCIe).  The host
    arrays are page-locked, as a caller that keeps its fields in pinned memory
    holds them; the library then moves them by DMA without a staging copy."""
    def pinned(a):
        t = torch.empty(a.shape, dtype=torch.float64).pin_memory()
        h = t.numpy()
        h[...] = a
        return t, h

    keep = [pinned(np.ascontiguousarray(a)) for a in (case_e.q, case_e.w, case_e.vhi, np.zeros_like(case_e.q))]
    q, w, vhi, qout = (h for _, h in keep)
    lib = s_e.lib
    ttc = C.c_double()
    barrier()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for k in range(steps):
        s_e._check(lib.upload(s_e.ctx, abi.dptr(q), abi.dptr(w), abi.dptr(vhi), 0.0), "upload")
        if sharded:
            s_e.dstep(k + 1, check=False)
        else:
            st = abi.Stats()
            lib.step(s_e.ctx, k + 1, C.byref(st))
        s_e._check(lib.download(s_e.ctx, abi.dptr(qout), None, None, C.byref(ttc)), "download")
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    units = case_e.ncells * iters_per_step(case_e) * steps * (1 if sharded else world)
    return {"value": units / e2e_s / 1e6, "unit": unit_of_case(case_e),
            "h2d_bytes_per_step": int(q.nbytes + w.nbytes + vhi.nbytes), "d2h_bytes_per_step": int(qout.nbytes)}


def accuracy_vs_oracle(args, q_orc, orc_status):
    """Relative L2 (all conserved variables, and the largest per-component
    value) of the GPU FP64 and mixed paths against the CPU restatement after the
    same args.cpu_steps steps from the same initial state."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import rel_l2, rel_l2_per_component
    from shared_cfd_b200.solver import Solver
    out = {"steps": args.cpu_steps, "oracle_status": orc_status}
    for prec, tag in ((abi.PREC_FP64, "fp64"), (abi.PREC_MIXED, "mixed")):
        case = make_case(args.config, args.scale, prec)
        s = Solver(case)
        s.upload()
        s.prepare(1)
        st = s.run(1, args.cpu_steps, check=False)
        q = s.download()[0]
        s.close()
        out[tag + "_vs_oracle"] = rel_l2(case, q, q_orc)
        out[tag + "_vs_oracle_per_component_max"] = rel_l2_per_component(case, q, q_orc)[0]
        out[tag + "_status"] = st.status
    return out


def controls_note(case):
    d = case.desc
    if d.scheme != abi.SCHEME_NR:
        return None
    return {"omega_max": d.omega_max, "omega_min": d.omega_min, "dqrate_max": d.dq_max,
            "res_rate_err": d.res_rate_err if d.res_rate_err < 1e299 else "off"}


if __name__ == "__main__":
    sys.exit(main())
