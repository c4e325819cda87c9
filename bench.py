"""Benchmark: successful cell-steps/s of the per-cell chemistry solve on B200.

Workload (default): the cb05cl_ae5 gas-phase mechanism (74 dependent species,
186 reactions) on 100 000 seeded synthetic cells per GPU, the 10-step
sequence of 60 s host steps, rtol 1e-4, atol 1e-8 ppm, the reference's
default limits (10 000 internal steps, 1 000 convergence / error-test
failures).  Cell states: T ~ U(260, 310) K, P ~ U(5e4, 1.013e5) Pa,
photolysis = 1e-4 s^-1 base set (jo2 = 0) x U[0,1], variable species
log-uniform 1e-6..1e2 ppm (seed 20241203).  No dataset exists for this path;
seeded synthetic cells with the workload's distributions stand in for it.

One bench "step" is one host time step: every cell advanced over 60 s by its
own BDF integration.  The sequence restarts from the seeded state every 10
steps (warm-up steps included).  About a quarter of these cells cannot
finish a host step under the reference's semantics (they end in
TOO_MUCH_WORK after 10 000 internal steps; see tests/test_hard_cells.py), so
value counts successful cell-steps only: cells that finished their host step
x steps / device time of the timed steps (CUDA events on the launch stream,
L2 flushed between steps), max over ranks; every cell-step, failed or not, is
reported beside it.  e2e = the same through solver_run with pinned host
buffers (host<->device copies inside the timed region, host clock) over the
first --e2e-steps steps of the sequence.

--impl reference times the reference's own C derivative/Jacobian code
(compiled from the reference sources into oracle/_ref) driven by the restated
CVODE BDF and sparse LU on all host cores, on a sample of 1 024 cells of the
same workload with the GPU arm's mix of host-step positions in the sequence.
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
# test/monarch/config_monarch_mod37.json as shipped (with the ZSR / PD-FiTE
# sub-models)
MOD37_SHIPPED_FILE = os.path.join(ROOT, "tests", "golden", "monarch_mod37_shipped.mech.json")
MECH_FILES = {"cb05cl_ae5": MECH_FILE, "monarch_mod37_shipped": MOD37_SHIPPED_FILE}
METRIC = "cell-steps/s (cb05, 1e5 cells) mixed vs FP64 GPU @rtol1e-4; p50/p99 column latency"
# DRAM bytes (read + write) per cell of one solve launch, from an ncu capture
# of the solve kernel on 2 000 cells (3.19 MB); the launch's traffic grows
# with the cells it processes
TRAFFIC_BYTES_PER_CELL = 2.833e6 / 2000
# nominal B200 FP64 (non-tensor) peak, for the algorithmic-flop fraction
FP64_PEAK_TFLOPS = 40.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cells", type=int, default=100000)
    ap.add_argument("--mech", default="cb05cl_ae5", choices=sorted(MECH_FILES),
                    help="mechanism of the main workload (cb05cl_ae5 is the metric's)")
    ap.add_argument("--dt", type=float, default=60.0)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--no-fp64-compare", action="store_true")
    ap.add_argument("--fp64-steps", type=int, default=3,
                    help="timed steps of the FP64 comparison (first steps of the sequence)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=3,
                    help="timed steps of the end-to-end measurement (first steps of the sequence)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample", type=int, default=1024,
                    help="cells of the reference arm's sample")
    ap.add_argument("--cpu-baseline-sample", type=int, default=256,
                    help="cells of the GPU arm's cpu_baseline sample")
    ap.add_argument("--cpu-one-core", type=int, default=24,
                    help="cells timed on one core for the single-core figure")
    ap.add_argument("--max-steps", type=int, default=10000)
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-mod37", action="store_true",
                    help="skip the mod37 blocks (gas phase; SOA; SOA + cloud partitioning)")
    ap.add_argument("--no-cost-order", action="store_true",
                    help="fetch cells in index order instead of longest-first")
    ap.add_argument("--no-graph", action="store_true",
                    help="launch the device step directly instead of as a CUDA graph")
    ap.add_argument("--serve-rates", default="5,10,20,30,40",
                    help="Poisson arrival rates (requests/s) of the serving sweep")
    ap.add_argument("--serve-seconds", type=float, default=8.0)
    ap.add_argument("--synth-cells", type=int, default=20000,
                    help="cells of the 200-species / 600-reaction synthetic mechanism (0: skip; "
                         "about a minute at 2e4 cells, five at 1e5)")
    ap.add_argument("--synth-dt", type=float, default=3.0,
                    help="host step of the synthetic mechanism (s): the longest at which the "
                         "oracle finishes every sampled cell")
    ap.add_argument("--synth-lane-cells", type=int, default=0,
                    help="cells of the lane-per-cell comparison on the synthetic mechanism "
                         "(0: skip; 11x slower than the block-per-cell kernel)")
    ap.add_argument("--serve-columns", type=int, default=256,
                    help="device-resident columns in the serving pool")
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
def sequence_positions(steps: int, warmup: int) -> list[int]:
    """Host-step position in the 10-step sequence of each timed step (the
    sequence restarts from the seeded state every 10 steps, warm-up steps
    included)."""
    return [(warmup + k) % 10 for k in range(steps)]


def cpu_sample_run(mech, n_sample, positions, dt, max_steps, one_core_cells):
    """Successful cell-steps/s of the CPU path on a sample of the workload:
    the first n_sample seeded cells of the GPU arm, cell i taken at host-step
    position positions[i % len(positions)] of the sequence (so the sample has
    the timed region's mix of positions and hard cells).  Each cell is first
    advanced, untimed, to its position (a cell that fails keeps its state, as
    solver_run leaves it, so it is not advanced again); then every cell's
    host step is timed as one job on all host cores (cells taken in chunks of
    8 by the threads) and, for the single-core figure, one_core_cells of
    them spread evenly over the sample on one thread."""
    from camp_b200.cells import make_cells
    from oracle.oracle import OracleModel, ref_available, ref_solve

    n_threads = os.cpu_count() or 1
    atol = np.full(mech.n_state_var, 1e-8)
    kind = "reference" if ref_available() else "port"
    om = None if kind == "reference" else OracleModel(mech)

    def solve(st, env, photo, threads):
        if kind == "reference":
            status, _ = ref_solve(mech, st, env, photo, 0.0, dt, 1e-4, atol, max_steps=max_steps,
                                  n_threads=threads, chunk=8)
            return status
        _, status, _, _ = om.solve(st, env, photo, 0.0, dt, 1e-4, atol, max_steps=max_steps,
                                   n_threads=threads)
        return status

    cells = make_cells(mech, n_sample, SEED)
    pos = np.asarray([positions[i % len(positions)] for i in range(n_sample)])
    state = cells.state.copy()
    stuck = np.zeros(n_sample, bool)
    for j in range(1, 10):
        idx = np.nonzero((pos >= j) & ~stuck)[0]
        if idx.size == 0:
            continue
        st = np.ascontiguousarray(state[idx])
        status = solve(st, cells.env[idx], cells.photo_rates[idx], n_threads)
        state[idx] = st
        stuck[idx[status != 0]] = True
    timed = state.copy()
    t0 = time.perf_counter()
    status = solve(timed, cells.env, cells.photo_rates, n_threads)
    wall = time.perf_counter() - t0
    ok = int(np.count_nonzero(status == 0))
    m = min(one_core_cells, n_sample)
    sel = np.linspace(0, n_sample - 1, m).astype(int)  # spread over the sample
    one = state[sel].copy()
    t0 = time.perf_counter()
    st1 = solve(one, cells.env[sel], cells.photo_rates[sel], 1)
    wall1 = time.perf_counter() - t0
    how = ("reference C f/J compiled from the reference sources + restated CVODE BDF / sparse LU"
           if kind == "reference" else
           "oracle C restatement of the reference f/J + restated CVODE BDF / sparse LU")
    return {
        "value": ok / wall,
        "unit": "cell-steps/s",
        "cores": n_threads,
        "kind": kind,
        "sample": (f"{n_sample} seeded cells of the workload, one host step of {dt:g} s each at "
                   f"the timed region's sequence positions {sorted(set(positions))}; "
                   f"successful cell-steps / wall time on {n_threads} threads; {how}"),
        "all_cell_steps_per_s": n_sample / wall,
        "ok_cell_fraction": ok / n_sample,
        "one_core": {"value": int(np.count_nonzero(st1 == 0)) / wall1, "cells": m,
                     "all_cell_steps_per_s": m / wall1},
        "wall_s": wall,
    }


def run_reference_arm(args):
    # the CPU arm needs no process group: rank 0 runs, the other ranks exit
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from camp_b200.mechanism import Mechanism

    mech = Mechanism.load(MECH_FILES[args.mech])
    positions = sequence_positions(args.steps, args.warmup)
    cb = cpu_sample_run(mech, args.cpu_sample, positions, args.dt, args.max_steps,
                        args.cpu_one_core)
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": cb["value"],
        "unit": "cell-steps/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * cb["wall_s"] / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "cb05cl_ae5, the GPU arm's seeded cells, host steps of 60 s "
                               "(10-step sequence), rtol 1e-4, atol 1e-8 ppm, max "
                               f"{args.max_steps} internal steps",
                   "cells_sampled": args.cpu_sample, "dt_s": args.dt, "seed": SEED},
        "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "all_cell_steps_per_s": cb["all_cell_steps_per_s"],
        "ok_cell_fraction": cb["ok_cell_fraction"],
        "one_core": cb["one_core"],
        "e2e": {"value": cb["value"], "unit": "cell-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Serving sweep
# ---------------------------------------------------------------------------
SERVE_P99_TARGET_MS = 2500.0  # stated p99 target of the serving loop


def serving_run(args, precision):
    """Open-loop Poisson arrivals of column steps at each rate against a pool
    of device-resident columns: 10-200 cells per column, 70 % cb05cl_ae5 and
    30 % MONARCH mod37 with its SOA scheme (cb05 + dry deposition,
    emissions, wet deposition and SIMPOL partitioning of the 2-product SOA
    into the modal/binned representation, the "monarch_mod37" of the
    workload); each arrival advances one column of the pool by a host step
    of 60, 300 or 900 s (a column's steps run in order, its concentrations
    stay on the device between them).  Latency is submit-to-completion inside
    the library.  Reported: p50 / p99 per offered rate, and the highest
    offered rate whose p99 stays within the stated target."""
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
    pool = []
    for k in range(args.serve_columns):
        mi = 0 if rng.uniform() < 0.7 else 1
        n = int(rng.integers(10, 201))
        c = make_cells(mechs[mi][0], n, int(rng.integers(1 << 30)), photo_base=mechs[mi][1])
        pool.append((mi, c, server.open_column(ids[mi], c.state)))
    clock = [0.0] * len(pool)  # each column's model time
    out = []
    for rate in [float(x) for x in args.serve_rates.split(",")]:
        arrivals = []
        t = 0.0
        while True:
            t += rng.exponential(1.0 / rate)
            if t > args.serve_seconds:
                break
            arrivals.append((t, int(rng.integers(len(pool))),
                             float(rng.choice([60.0, 300.0, 900.0]))))
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
        for (ta, k, dt) in arrivals:
            delay = t0 + ta - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            mi, c, cid = pool[k]
            rid = server.submit_column(cid, c.env, c.photo_rates, clock[k], clock[k] + dt)
            clock[k] += dt
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
    for _, _, cid in pool:
        server.close_column(cid)
    server.close()
    for s in solvers:
        s.free()
    held = [r["offered_rps"] for r in out if r["p99_ms"] <= SERVE_P99_TARGET_MS]
    return {"mix": "70% cb05cl_ae5 / 30% monarch_mod37 with SOA (cb05 + dry deposition, "
                   "emissions, wet deposition, SIMPOL partitioning into the modal/binned "
                   f"representation); pool of {len(pool)} device-resident columns of 10-200 "
                   "cells; each arrival one host step of 60/300/900 s of a random column; "
                   "Poisson arrivals",
            "precision": "mixed" if precision == 1 else "fp64", "slots": 8,
            "seconds_per_rate": args.serve_seconds,
            "p99_target_ms": SERVE_P99_TARGET_MS,
            "max_rate_within_p99_target": max(held) if held else None,
            "rates": out}


# ---------------------------------------------------------------------------
# Algorithmic flops
# ---------------------------------------------------------------------------
def flop_model(mech, solver) -> dict:
    """Flops of each counted operation of one cell, from the mechanism and
    the solver's sparsity and elimination order: f (rate = k x reactants,
    one add per loss or gain, one multiply per yield, P - L per species), J
    (the partials and their gathers, 2 nr (nr + np) per reaction), the LU of
    M = I - gamma J (2 per Schur update, 1 per L scaling, 1 reciprocal per
    pivot, 2 per entry of M), one solve (2 per LU entry) and the BDF vector
    work of one internal step (prediction, Newton updates, norms, error
    test, history update: about 30 per dependent species)."""
    f = j = 0
    for r in mech.rxns:
        nr, npd = int(r.ints[0]), int(r.ints[1])
        f += nr + nr + 2 * npd
        j += 2 * nr * (nr + npd)
    n = mech.n_dep_var
    f += n
    cp, ri = solver.solver_jac()
    perm = solver.lu_order()
    pos = np.empty(n, int)
    pos[perm] = np.arange(n)
    rows = [set() for _ in range(n)]  # pattern in pivot order, by row
    for c in range(n):
        for r in ri[cp[c]:cp[c + 1]]:
            rows[pos[r]].add(pos[c])
    for i in range(n):
        rows[i].add(i)
    upd = scal = 0
    for k in range(n):  # right-looking symbolic elimination
        urow = [c for c in rows[k] if c > k]
        for i in range(k + 1, n):
            if k in rows[i]:
                scal += 1
                upd += len(urow)
                rows[i].update(urow)
    nnz = sum(len(r) for r in rows)
    return {"f": f, "jac": j, "lu": 2 * upd + scal + n + 2 * nnz, "solve": 2 * nnz,
            "bdf_step": 30 * n, "lu_entries": nnz, "lu_entries_solver": solver.n_lu()}


def counted_flops(model: dict, stats) -> float:
    """Flops of the operations the per-cell counters recorded."""
    return float(model["f"] * stats["nfe"].sum() + model["jac"] * stats["nje"].sum()
                 + model["lu"] * stats["nsetups"].sum() + model["solve"] * stats["nni"].sum()
                 + model["bdf_step"] * stats["nst"].sum())


# ---------------------------------------------------------------------------
# First host step of other mechanisms
# ---------------------------------------------------------------------------
def run_first_step(mech, args, dev, stream, n, cells=None, dt=None, kernel=None, reps=2):
    """n seeded cells of another mechanism over the first host step of the
    sequence (every cell from its seeded state), mixed and FP64,
    device-resident; with reps=2 longest-first order from a previous
    identical run, device time of the second run (reps=1: one run in seeded
    order).  kernel: camp_b200_set_kernel's value (None: the mechanism's
    default)."""
    import torch

    from camp_b200.cells import make_cells
    from camp_b200.solver import FP64, MIXED, Solver

    cells = cells if cells is not None else make_cells(mech, n, SEED)
    dt = args.dt if dt is None else dt
    init = torch.from_numpy(cells.state).to(dev)
    env = torch.from_numpy(cells.env).to(dev)
    photo = torch.from_numpy(np.ascontiguousarray(cells.photo_rates)).to(dev)
    out = {"mechanism": mech.name, "cells": n, "host_step_s": dt,
           "note": ("first host step of the sequence, cells ordered longest-first from an "
                    "identical previous run; device time (CUDA events)") if reps > 1 else
                   "first host step of the sequence, seeded cell order; device time (CUDA "
                   "events)"}
    for name, p in (("mixed", MIXED), ("fp64", FP64)):
        s = Solver(mech, n)
        s.initialize(abs_tol=np.full(mech.n_state_var, 1e-8), rel_tol=1e-4,
                     max_steps=args.max_steps)
        s.set_precision(p)
        if kernel is not None:
            s.set_kernel(kernel)
        out["kernel"] = s.kernel()
        s.set_photo_rates_device(photo, n)
        s.set_cost_ordering(reps > 1)
        s.set_graph(not args.no_graph)
        for rep in range(reps):
            st = init.clone()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            s.launch_device(st, env, n, 0.0, dt, stream)
            e1.record(stream)
            s.sync_status(stream)
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        st = s.cell_stats(n)
        ok = int(np.count_nonzero(st["status"] == 0))
        out[name] = {"ok_cell_steps_per_s": ok / (ms / 1e3),
                     "cell_steps_per_s": n / (ms / 1e3),
                     "internal_steps_per_s": int(st["nst"].sum()) / (ms / 1e3),
                     "ms": ms, "ok_cell_fraction": ok / n}
        s.free()
    out["mixed_over_fp64"] = (out["mixed"]["ok_cell_steps_per_s"]
                              / out["fp64"]["ok_cell_steps_per_s"])
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

    mech = Mechanism.load(MECH_FILES[args.mech])
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
    stat_keys = ("nst", "nfe", "nje", "nsetups", "nni")

    def device_run(s, steps, warmup):
        """warmup + timed host steps on device-resident inputs."""
        d_state = init_state.clone()
        # every input resident in HBM: photolysis rates from device memory too
        s.set_photo_rates_device(d_photo, n)
        step_ms, kernel_ms, ok_cells, launches0 = [], [], [], None
        counters = {k: 0 for k in stat_keys}
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
                for k in stat_keys:
                    counters[k] += int(st[k].sum())
        torch.cuda.synchronize()
        barrier(world)
        launches = s.kernel_launches() - launches0
        return step_ms, kernel_ms, ok_cells, launches, counters

    prec = MIXED if args.precision == "mixed" else FP64
    solver = make_solver(prec)
    with ClockSampler(local) as clk:
        step_ms, kernel_ms, ok_cells, launches, counters = device_run(solver, args.steps,
                                                                      args.warmup)
    total_s = max_over_ranks(sum(step_ms) / 1e3, world)
    ok_total = replicas.sum_over_ranks(sum(ok_cells), world)
    value = ok_total / total_s
    all_value = replicas.aggregate_throughput(n, args.steps, world, total_s)
    fp64 = None
    if not args.no_fp64_compare:
        k64 = min(args.fp64_steps, args.steps)
        s64 = make_solver(FP64)
        sm64, km64, ok64, _, c64 = device_run(s64, k64, 1)
        t64 = max_over_ranks(sum(sm64) / 1e3, world)
        ok64_total = replicas.sum_over_ranks(sum(ok64), world)
        # the mixed form over the same first steps of the sequence
        same = min(k64, args.steps)
        fp64 = {"value": ok64_total / t64,
                "unit": "cell-steps/s",
                "steps": k64,
                "ms_per_step": 1e3 * t64 / k64,
                "all_cell_steps_per_s": replicas.aggregate_throughput(n, k64, world, t64),
                "ok_cell_fraction": float(np.mean(ok64)) / n,
                "note": f"first {k64} timed steps of the sequence after 1 warm-up step"}
        s64.free()
        # the mixed form over the same sequence positions, for the ratio
        sm_m, _, ok_m, _, _ = device_run(solver, k64, 1)
        tm = max_over_ranks(sum(sm_m) / 1e3, world)
        okm_total = replicas.sum_over_ranks(sum(ok_m), world)
        fp64["mixed_same_steps"] = okm_total / tm
        fp64["mixed_over_fp64"] = fp64["mixed_same_steps"] / fp64["value"]
    e2e = None
    if not args.no_e2e:
        ke = min(args.e2e_steps, args.steps)
        # pinned host buffers; copies inside the timed region
        h_state = torch.empty((n, mech.n_state_var), dtype=torch.float64, pin_memory=True)
        h_env = torch.from_numpy(cells.env).pin_memory()
        hs, he = h_state.numpy(), h_env.numpy()
        # end to end: photolysis rates travel from the host with each run
        solver.set_photo_rates_device(None)
        times, oks = [], []
        for it in range(1 + ke):
            if it % 10 == 0 or it == 1:
                hs[:] = cells.state  # warm-up, then the sequence from its start
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            solver.solve(hs, he, 0.0, args.dt)
            if it >= 1:
                times.append(time.perf_counter() - t0)
                oks.append(int(np.count_nonzero(solver.cell_stats(n)["status"] == 0)))
        te = max_over_ranks(sum(times), world)
        n_photo = solver.n_photo
        e2e = {"value": replicas.sum_over_ranks(sum(oks), world) / te,
               "unit": "cell-steps/s",
               "h2d_bytes_per_step": int(8 * n * (mech.n_state_var + 2 + n_photo)),
               "d2h_bytes_per_step": int(8 * n * mech.n_state_var + 56 * n),
               "steps": ke,
               "all_cell_steps_per_s": replicas.aggregate_throughput(n, ke, world, te),
               "note": f"solver_run on pinned host buffers, first {ke} steps of the sequence "
                       "after 1 warm-up step, host clock"}
    serving = None
    if world == 1 and not args.no_serving:
        serving = {"mixed": serving_run(args, MIXED), "fp64": serving_run(args, FP64)}
    mod37 = mod37_soa = mod37_aero = mod37_shipped = None
    if world == 1 and not args.no_mod37:
        mod37 = run_first_step(Mechanism.load(MOD37_FILE), args, dev, stream, 10000)
        mod37_soa = run_first_step(Mechanism.load(MOD37_SOA_FILE), args, dev, stream, 10000)
        mod37_aero = run_first_step(Mechanism.load(MOD37_AERO_FILE), args, dev, stream, 10000)
        mod37_shipped = run_first_step(Mechanism.load(MOD37_SHIPPED_FILE), args, dev, stream,
                                       10000)
    synth = None
    if world == 1 and args.synth_cells > 0:
        # the seeded 200-species / 600-reaction mechanism on its default
        # (block-per-cell) kernel, and the lane-per-cell kernel on a smaller
        # sample, at the host step every sampled oracle cell finishes (its
        # cells gain molecules in every reaction: at 300 s none finishes)
        import tempfile

        from camp_b200.cells import make_cells
        from camp_b200.synth import load_synthetic

        with tempfile.TemporaryDirectory() as td:
            smech, sbase = load_synthetic(td, 200, 600)
        scells = make_cells(smech, args.synth_cells, SEED, conc_lo=1e-8, photo_base=sbase)
        synth = run_first_step(smech, args, dev, stream, args.synth_cells, cells=scells,
                               dt=args.synth_dt, reps=1)
        if args.synth_lane_cells > 0:
            nl = min(args.synth_lane_cells, args.synth_cells)
            lcells = make_cells(smech, nl, SEED, conc_lo=1e-8, photo_base=sbase)
            synth["lane_kernel"] = run_first_step(smech, args, dev, stream, nl, cells=lcells,
                                                  dt=args.synth_dt, kernel=1, reps=1)
    fm = flop_model(mech, solver)
    if rank != 0:
        solver.free()
        replicas.finalize(world)
        return
    cb = None
    if world == 1 and not args.no_cpu_baseline:
        cb = cpu_sample_run(mech, args.cpu_baseline_sample,
                            sequence_positions(args.steps, args.warmup), args.dt,
                            args.max_steps, args.cpu_one_core)
        cb = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample", "one_core",
                                 "ok_cell_fraction")}
    bpcs = bytes_per_cell_step(mech)
    mean_kernel_s = float(np.mean(kernel_ms)) / 1e3
    achieved = bpcs * n / mean_kernel_s / 1e9
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    flops = counted_flops(fm, {k: np.asarray([counters[k]]) for k in stat_keys})
    tflops = flops / (sum(kernel_ms) / 1e3) / 1e12
    internal = counters["nst"]
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
            "workload": f"{args.mech}, {n} cells per GPU, host steps of {args.dt:g} s "
                        "(10-step sequence), rtol 1e-4, atol 1e-8 ppm, max "
                        f"{args.max_steps} internal steps; value counts cells that finish "
                        "their host step",
            "cells_per_gpu": n, "dt_s": args.dt, "precision": args.precision,
            "l2": "flushed (256 MB write) before every timed step",
            "seed": SEED,
        },
        "all_cell_steps_per_s": all_value,
        "ok_cell_fraction": float(np.mean(ok_cells)) / n,
        "internal_steps_per_cell_step": internal / (n * args.steps),
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
                    "2000-cell capture.  HBM is not what bounds this kernel: see issue_bound",
        },
        "issue_bound": {
            "bound": "dependent-issue latency (warp per cell, cells resident in shared memory)",
            "achieved_fp64_tflops": tflops,
            "peak_fp64_tflops_nominal": FP64_PEAK_TFLOPS,
            "flop_frac": tflops / FP64_PEAK_TFLOPS,
            "flops_per_internal_step": flops / max(internal, 1),
            "internal_steps_per_s": internal / (sum(kernel_ms) / 1e3),
            "flop_model": fm,
            "note": "algorithmic flops of the counted f / J / LU / solve / BDF-step operations "
                    "(per-cell device counters) / kernel time, against the nominal FP64 peak; "
                    "ncu: IPC ~1.0 of 4, FP64 pipe ~4 %, warp stalls on fixed-latency "
                    "dependencies and shared-memory loads",
        },
        "cpu_baseline": cb,
        "serving": serving,
        "mod37_gas": mod37,
        "mod37_soa": mod37_soa,
        "mod37_aero": mod37_aero,
        "mod37_shipped": mod37_shipped,
        "synthetic_200sp_600rxn": synth,
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
