"""Benchmark: cell-steps/s of the per-cell chemistry solve on B200.

Workload (default): the cb05cl_ae5 gas-phase mechanism (74 dependent species,
186 reactions) on 10 000 seeded synthetic cells (--cells 100000 for the 1e5
case; the persistent kernel keeps every SM busy from ~2 000 cells up, so the
throughput per cell-step is the same), host steps of 60 s, rtol
1e-4, atol 1e-8 ppm, the reference's default limits (10 000 internal steps,
1 000 convergence / error-test failures).  Cell states: T ~ U(260, 310) K,
P ~ U(5e4, 1.013e5) Pa, photolysis = 1e-4 s^-1 base set (jo2 = 0) x U[0,1],
variable species log-uniform 1e-6..1e2 ppm (seed 20241203).

One bench "step" is one host time step: every cell advanced over 60 s by its
own BDF integration.  The 10-step sequence of the workload restarts from the
seeded initial state every 10 steps.  value = cells x steps / device time of
the timed steps (CUDA events on the launch stream, L2 flushed between steps),
max over ranks; e2e = the same through solver_run with pinned host buffers
(host<->device copies inside the timed region, host clock).

--impl reference times the reference's own C derivative/Jacobian code
(compiled from the reference sources into oracle/_ref) driven by the restated
CVODE BDF and sparse LU on all host cores, on a bounded sample of the same
workload (the same 10-step sequence for a subset of the cells).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SEED = 20241203
MECH_FILE = os.path.join(ROOT, "tests", "golden", "cb05cl_ae5.mech.json")
# gas phase of MONARCH mod37 (cb05 + dry deposition + emissions + the wet
# deposition of its cloud-and-rain phase), packed from the shipped files
MOD37_FILE = os.path.join(ROOT, "tests", "golden", "monarch_mod37_gas.mech.json")
# the same with the shipped 2-product SOA scheme (SIMPOL partitioning into the
# modal/binned aerosol representation), and with the partitioning of 35 gas
# species into cloud and rain water (HL) as well
MOD37_SOA_FILE = os.path.join(ROOT, "tests", "golden", "monarch_mod37_soa.mech.json")
MOD37_AERO_FILE = os.path.join(ROOT, "tests", "golden", "monarch_mod37_aero.mech.json")
# compulsory HBM bytes per cell-step of cb05cl_ae5: state read (80 x 8),
# env (16), photolysis base rates (25 x 8), dependent state write (74 x 8)
METRIC = "cell-steps/s (cb05, 1e5 cells) mixed vs FP64 GPU @rtol1e-4; p50/p99 column latency"
# DRAM bytes (read + write) per cell of one solve launch, from the ncu capture
# summarised in profiles/solve_kernel_mixed_cb05_2000cells.md (3.19 MB for
# 2 000 cells); the launch's traffic grows with the cells it processes
TRAFFIC_BYTES_PER_CELL = 3.187e6 / 2000


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cells", type=int, default=10000)
    ap.add_argument("--dt", type=float, default=60.0)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--no-fp64-compare", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample", type=int, default=128)
    ap.add_argument("--max-steps", type=int, default=10000)
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-1e5", action="store_true",
                    help="skip the 1e5-cell single-host-step measurement")
    ap.add_argument("--no-mod37", action="store_true",
                    help="skip the mod37 blocks (gas phase; SOA; SOA + cloud partitioning)")
    ap.add_argument("--no-cost-order", action="store_true",
                    help="fetch cells in index order instead of longest-first")
    ap.add_argument("--no-graph", action="store_true",
                    help="launch the device step directly instead of as a CUDA graph")
    ap.add_argument("--serve-rates", default="5,10,20,40",
                    help="Poisson arrival rates (requests/s) of the serving sweep")
    ap.add_argument("--serve-seconds", type=float, default=8.0)
    return ap.parse_args()


def bytes_per_cell_step(mech) -> int:
    n_rates = len(mech.rate_rxns())  # host-set base rates per cell
    return 8 * mech.n_state_var + 16 + 8 * n_rates + 8 * mech.n_dep_var


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            for n, v in zip(names, s[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def dist_init():
    from camp_b200 import replicas

    return replicas.init("nccl")


def max_over_ranks(x: float, world: int) -> float:
    from camp_b200 import replicas

    return replicas.max_over_ranks(x, world)


def barrier(world):
    from camp_b200 import replicas

    replicas.barrier(world)


# ---------------------------------------------------------------------------
# CPU reference arm
# ---------------------------------------------------------------------------
def cpu_reference_run(mech, cells, steps, warmup, dt, sample, max_steps):
    """Times the reference's C f/J + restated BDF on all host cores; each step
    is the same host step of the 10-step sequence for `sample` cells."""
    from oracle.oracle import ref_available, ref_solve, OracleModel

    n_threads = os.cpu_count() or 1
    atol = np.full(mech.n_state_var, 1e-8)
    kind = "reference" if ref_available() else "port"
    sub = cells.slice(0, sample)
    state = sub.state.copy()
    times = []
    om = None if kind == "reference" else OracleModel(mech)
    for it in range(warmup + steps):
        if it % 10 == 0:
            state = sub.state.copy()
        t0 = time.perf_counter()
        if kind == "reference":
            ref_solve(mech, state, sub.env, sub.photo_rates, 0.0, dt, 1e-4, atol,
                      max_steps=max_steps, n_threads=n_threads)
        else:
            om.solve(state, sub.env, sub.photo_rates, 0.0, dt, 1e-4, atol,
                     max_steps=max_steps, n_threads=n_threads)
        if it >= warmup:
            times.append(time.perf_counter() - t0)
    per_step = float(np.mean(times))
    return {
        "value": sample / per_step,
        "unit": "cell-steps/s",
        "cores": n_threads,
        "kind": kind,
        "sample": (f"{sample} cells x {steps} host steps of {dt:g} s (the workload's 10-step "
                   f"sequence for the first {sample} seeded cells); "
                   + ("reference C f/J compiled from the reference sources + restated "
                      "CVODE BDF / sparse LU" if kind == "reference" else
                      "oracle C restatement of the reference f/J + restated CVODE BDF / sparse LU")),
        "ms_per_step": per_step * 1e3,
    }


def run_reference_arm(args):
    # the CPU arm needs no process group: rank 0 runs, the other ranks exit
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from camp_b200.cells import make_cells
    from camp_b200.mechanism import Mechanism

    mech = Mechanism.load(MECH_FILE)
    cells = make_cells(mech, args.cpu_sample, SEED)
    cb = cpu_reference_run(mech, cells, args.steps, args.warmup, args.dt, args.cpu_sample,
                           args.max_steps)
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": cb["value"],
        "unit": "cell-steps/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": cb["ms_per_step"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "cb05cl_ae5 cell states, host steps of 60 s, rtol 1e-4, atol 1e-8 ppm",
                   "cells_per_step": args.cpu_sample, "dt_s": args.dt},
        "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": cb["value"], "unit": "cell-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Serving sweep
# ---------------------------------------------------------------------------
def serving_run(args, precision):
    """Open-loop Poisson arrivals of column requests at each rate: 10-200
    cells per column, 70 % cb05cl_ae5 and 30 % MONARCH mod37 with its SOA
    scheme (dry deposition, emissions, wet deposition and SIMPOL partitioning
    into the modal/binned representation, per-cell mode GMD / GSD), host
    steps of 60, 300 or 900 s.  Latency is submit-to-completion inside the
    library."""
    from camp_b200.cells import make_cells, photo_base_rates
    from camp_b200.mechanism import Mechanism
    from camp_b200.serve import Server
    from camp_b200.solver import Solver

    cb05 = Mechanism.load(MECH_FILE)
    mod37 = Mechanism.load(MOD37_SOA_FILE)
    mechs = [(cb05, photo_base_rates(cb05)), (mod37, photo_base_rates(mod37))]
    solvers = []
    for m, _ in mechs:
        s = Solver(m, 200)
        s.initialize(abs_tol=np.full(m.n_state_var, 1e-8), rel_tol=1e-4,
                     max_steps=args.max_steps)
        s.set_precision(precision)
        solvers.append(s)
    server = Server(n_slots=8, device_mb=4096, host_mb=1024)
    ids = [server.add_solver(s) for s in solvers]
    rng = np.random.Generator(np.random.PCG64(SEED + 1))
    out = []
    for rate in [float(x) for x in args.serve_rates.split(",")]:
        arrivals = []
        t = 0.0
        while True:
            t += rng.exponential(1.0 / rate)
            if t > args.serve_seconds:
                break
            mi = 0 if rng.uniform() < 0.7 else 1
            n = int(rng.integers(10, 201))
            dt = float(rng.choice([60.0, 300.0, 900.0]))
            c = make_cells(mechs[mi][0], n, int(rng.integers(1 << 30)), photo_base=mechs[mi][1])
            arrivals.append((t, mi, c, dt))
        results = []

        def collect(q):
            while True:
                item = q.get()
                if item is None:
                    return
                rid, n = item
                rc, ms, _, _ = server.wait(rid)
                results.append((ms, n, time.perf_counter()))

        import queue

        q = queue.Queue()
        th = threading.Thread(target=collect, args=(q,), daemon=True)
        th.start()
        t0 = time.perf_counter()
        for (ta, mi, c, dt) in arrivals:
            delay = t0 + ta - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            rid = server.submit(ids[mi], c.state, c.env, c.photo_rates, 0.0, dt)
            q.put((rid, c.n_cells))
        q.put(None)
        th.join()
        lat = np.array([r[0] for r in results])
        cells = sum(r[1] for r in results)
        span = max(r[2] for r in results) - t0
        out.append({"offered_rps": rate, "requests": len(results),
                    "achieved_rps": len(results) / span, "cells_per_s": cells / span,
                    "p50_ms": float(np.percentile(lat, 50)),
                    "p99_ms": float(np.percentile(lat, 99))})
    server.close()
    for s in solvers:
        s.free()
    return {"mix": "70% cb05cl_ae5 / 30% monarch_mod37 with SOA (cb05 + dry deposition, "
                   "emissions, wet deposition, SIMPOL partitioning into the modal/binned "
                   "representation); 10-200 cells; host steps 60/300/900 s; Poisson arrivals",
            "precision": "mixed" if precision == 1 else "fp64", "slots": 8,
            "seconds_per_rate": args.serve_seconds, "rates": out}


# ---------------------------------------------------------------------------
# 1e5 cells, one host step
# ---------------------------------------------------------------------------
def run_1e5(mech, args, dev, stream, n=100000):
    """The metric's cell count: 1e5 seeded cells over the first host step of
    the sequence (the most expensive one: every cell starts from its seeded
    state), mixed and FP64, device-resident, longest-first order from a
    previous identical run; device time of the second run.  Also used with
    another mechanism and cell count for the mod37 blocks."""
    import torch

    from camp_b200.cells import make_cells
    from camp_b200.solver import FP64, MIXED, Solver

    cells = make_cells(mech, n, SEED)
    init = torch.from_numpy(cells.state).to(dev)
    env = torch.from_numpy(cells.env).to(dev)
    photo = torch.from_numpy(np.ascontiguousarray(cells.photo_rates)).to(dev)
    out = {"mechanism": mech.name, "cells": n, "host_step_s": args.dt,
           "note": "first host step of the sequence, cells ordered longest-first from an "
                   "identical previous run; device time (CUDA events)"}
    for name, p in (("mixed", MIXED), ("fp64", FP64)):
        s = Solver(mech, n)
        s.initialize(abs_tol=np.full(mech.n_state_var, 1e-8), rel_tol=1e-4,
                     max_steps=args.max_steps)
        s.set_precision(p)
        s.set_photo_rates_device(photo, n)
        s.set_cost_ordering(True)
        s.set_graph(not args.no_graph)
        for rep in range(2):
            st = init.clone()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            s.launch_device(st, env, n, 0.0, args.dt, stream)
            e1.record(stream)
            s.sync_status(stream)
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        st = s.cell_stats(n)
        nst = int(st["nst"].sum())
        out[name] = {"cell_steps_per_s": n / (ms / 1e3), "internal_steps_per_s": nst / (ms / 1e3),
                     "ms": ms, "ok_cell_fraction": float(np.mean(st["status"] == 0))}
        s.free()
    out["mixed_over_fp64"] = out["mixed"]["cell_steps_per_s"] / out["fp64"]["cell_steps_per_s"]
    return out


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def run_gpu_arm(args):
    world, rank, local = dist_init()
    import torch

    torch.cuda.set_device(local)
    from camp_b200.cells import make_cells
    from camp_b200.mechanism import Mechanism
    from camp_b200.solver import FP64, MIXED, Solver

    mech = Mechanism.load(MECH_FILE)
    n = args.cells
    from camp_b200 import replicas

    cells = make_cells(mech, n, replicas.rank_seed(SEED, rank))
    atol = np.full(mech.n_state_var, 1e-8)
    dev = torch.device("cuda", local)
    # a created stream: the legacy default stream (handle 0) would read as
    # "the solver's own stream" at the C ABI
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def make_solver(prec):
        s = Solver(mech, n)
        s.initialize(abs_tol=atol, rel_tol=1e-4, max_steps=args.max_steps)
        s.set_precision(prec)
        s.set_photo_rates(cells.photo_rates)
        # device step (counter reset + solve kernel) as one CUDA graph
        s.set_graph(not args.no_graph)
        # persistent-kernel schedule: cells in decreasing order of their
        # internal step count in the previous host step (longest first)
        s.set_cost_ordering(not args.no_cost_order)
        return s

    init_state = torch.from_numpy(cells.state).to(dev)
    d_env = torch.from_numpy(cells.env).to(dev)
    d_photo = torch.from_numpy(np.ascontiguousarray(cells.photo_rates)).to(dev)

    def device_run(s, steps, warmup):
        """warmup + timed host steps on device-resident inputs."""
        d_state = init_state.clone()
        # every input resident in HBM: photolysis rates from device memory too
        s.set_photo_rates_device(d_photo, n)
        step_ms, ok_cells, launches0 = [], [], None
        kernel_ms = []
        for it in range(warmup + steps):
            if it % 10 == 0:
                d_state.copy_(init_state)
            flush.zero_()
            if it == warmup:
                barrier(world)
                torch.cuda.synchronize()
                launches0 = s.kernel_launches()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            s.launch_device(d_state, d_env, n, 0.0, args.dt, stream)
            e1.record(stream)
            s.sync_status(stream)
            if it >= warmup:
                torch.cuda.synchronize()
                step_ms.append(e0.elapsed_time(e1))
                kernel_ms.append(s.last_kernel_ms())
                st = s.cell_stats(n)
                ok_cells.append(int(np.count_nonzero(st["status"] == 0)))
        torch.cuda.synchronize()
        barrier(world)
        launches = s.kernel_launches() - launches0
        return step_ms, kernel_ms, ok_cells, launches, s.cell_stats(n)

    prec = MIXED if args.precision == "mixed" else FP64
    solver = make_solver(prec)
    with ClockSampler(local) as clk:
        step_ms, kernel_ms, ok_cells, launches, last_stats = device_run(solver, args.steps, args.warmup)
    total_s = max_over_ranks(sum(step_ms) / 1e3, world)
    value = replicas.aggregate_throughput(n, args.steps, world, total_s)
    fp64 = None
    if not args.no_fp64_compare:
        s64 = make_solver(FP64)
        sm64, km64, ok64, _, _ = device_run(s64, args.steps, min(args.warmup, 3))
        t64 = max_over_ranks(sum(sm64) / 1e3, world)
        fp64 = {"value": replicas.aggregate_throughput(n, args.steps, world, t64),
                "unit": "cell-steps/s",
                "ms_per_step": 1e3 * t64 / args.steps,
                "ok_cell_fraction": float(np.mean(ok64)) / n}
        s64.free()
    e2e = None
    if not args.no_e2e:
        # pinned host buffers; copies inside the timed region
        h_state = torch.empty((n, mech.n_state_var), dtype=torch.float64, pin_memory=True)
        h_env = torch.from_numpy(cells.env).pin_memory()
        hs, he = h_state.numpy(), h_env.numpy()
        # end to end: photolysis rates travel from the host with each run
        solver.set_photo_rates_device(None)
        times = []
        for it in range(args.warmup + args.steps):
            if it % 10 == 0:
                hs[:] = cells.state
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            solver.solve(hs, he, 0.0, args.dt)
            if it >= args.warmup:
                times.append(time.perf_counter() - t0)
        te = max_over_ranks(sum(times), world)
        n_photo = solver.n_photo
        e2e = {"value": replicas.aggregate_throughput(n, args.steps, world, te),
               "unit": "cell-steps/s",
               "h2d_bytes_per_step": int(8 * n * (mech.n_state_var + 2 + n_photo)),
               "d2h_bytes_per_step": int(8 * n * mech.n_state_var + 56 * n)}
    serving = None
    if world == 1 and not args.no_serving:
        serving = serving_run(args, prec)
    at_1e5 = None
    if world == 1 and not args.no_1e5:
        at_1e5 = run_1e5(mech, args, dev, stream)
    mod37 = mod37_soa = mod37_aero = None
    if world == 1 and not args.no_mod37:
        mod37 = run_1e5(Mechanism.load(MOD37_FILE), args, dev, stream, n=10000)
        mod37_soa = run_1e5(Mechanism.load(MOD37_SOA_FILE), args, dev, stream, n=10000)
        mod37_aero = run_1e5(Mechanism.load(MOD37_AERO_FILE), args, dev, stream, n=10000)
    if rank != 0:
        solver.free()
        replicas.finalize(world)
        return
    cb = None
    if world == 1 and not args.no_cpu_baseline:
        cpu_cells = make_cells(mech, args.cpu_sample, SEED)
        cb = cpu_reference_run(mech, cpu_cells, min(args.steps, 10), 1, args.dt, args.cpu_sample,
                               args.max_steps)
        cb = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
    bpcs = bytes_per_cell_step(mech)
    mean_kernel_s = float(np.mean(kernel_ms)) / 1e3
    achieved = bpcs * n / mean_kernel_s / 1e9
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "cell-steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * total_s / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64+f32 (mixed: FP32 Jacobian/LU, FP64 residual/state/error test)"
                 if prec == MIXED else "f64",
        "data": "synthetic",
        "config": {
            "workload": f"cb05cl_ae5, {n} cells per GPU, host steps of {args.dt:g} s "
                        "(10-step sequence), rtol 1e-4, atol 1e-8 ppm, max "
                        f"{args.max_steps} internal steps",
            "cells_per_gpu": n, "dt_s": args.dt, "precision": args.precision,
            "l2": "flushed (256 MB write) before every timed step",
            "seed": SEED,
        },
        "ok_cell_fraction": float(np.mean(ok_cells)) / n,
        "internal_steps_per_cell_step": float(np.mean(last_stats["nst"])),
        "fp64": fp64,
        "e2e": e2e,
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "roofline": {
            "bound": "hbm",
            "achieved": achieved,
            "peak": peak,
            "unit": "GB/s",
            "frac": achieved / peak,
            "traffic": TRAFFIC_BYTES_PER_CELL * n,
            "note": f"{bpcs} compulsory bytes per cell-step x cells / mean solve-kernel time "
                    "(of measured peak); traffic = ncu DRAM bytes per launch scaled from a "
                    "2000-cell capture; the kernel is bound by dependent-issue latency (IPC "
                    "1.0, FP64 pipe 4.4 %, profiles/solve_kernel_mixed_cb05_2000cells.md), "
                    "not by HBM",
        },
        "cpu_baseline": cb,
        "serving": serving,
        "cells_1e5": at_1e5,
        "mod37_gas": mod37,
        "mod37_soa": mod37_soa,
        "mod37_aero": mod37_aero,
    }
    print(json.dumps(line), flush=True)
    solver.free()
    replicas.finalize(world)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_gpu_arm(args)


if __name__ == "__main__":
    main()
