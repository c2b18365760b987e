"""Benchmark: steady SIMPLE (k-omega SST, plain FP64) on NACA 0012 C-grids.

Workload (one "step" = one SIMPLE outer iteration of every solve in it):
  NACA 0012, Re 1e6, k-omega SST, inflow intensity 0.1 %, mu_t/mu 10,
  medium C-grid 384 x 96 cells (surface 128, wake 65, normal 97 points;
  upstream/vertical 10 chords, downstream 15; first layer 1e-5 chord),
  two solves at alpha 0 deg and 4 deg in one batched launch. Synthetic inputs:
  the uniform freestream start of FlowField::uniform, advanced by the warm-up
  steps; no dataset exists for this path.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0). `value` is cell-iterations/s over all ranks,
timed with CUDA events around each step's launch on the launching stream; L2
(126 MB) is flushed between timed steps by writing a 256 MiB buffer. `e2e` is
the same metric through the C ABI from pinned host buffers: each step loads
the solver state host->device, iterates once, and reads the monitors back.
`--impl reference` times the reference's own CPU solver (compiled from its
sources into oracle/_ref) on the same workload with every host core.
Multi-GPU (torchrun): independent replicas, one per GPU; no collective on the
data path (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "cfd-simulator_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "SIMPLE cell-iters/s, % HBM roofline; solves/min + p99, mixed vs FP64 at ΔCl≤1e-4"
UNIT = "cell-iters/s"
WORKLOAD = dict(designation="0012", surface_points=128, wake_points=65, normal_points=97,
                first_layer_height=1e-5, upstream_chords=10.0, downstream_chords=15.0,
                vertical_chords=10.0)
ALPHAS = (0.0, 4.0)
REYNOLDS = 1e6
INTENSITY = 0.001
VISCOSITY_RATIO = 10.0


def config(extra=None):
    c = {"workload": "NACA0012 k-omega SST Re1e6 C-grid 384x96 (medium), alpha 0 and 4 deg, "
                     "plain FP64, batched in one launch",
         "cells_per_solve": 384 * 96, "solves": len(ALPHAS), "model": "k-omega SST",
         "precision": "fp64 plain (reference-parity form)",
         "l2": "flushed between timed steps (256 MiB write)", "parallelism": "replicas"}
    if extra:
        c.update(extra)
    return c


# ---------------------------------------------------------------- clocks ---

class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during timing."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        mhz, maxes, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                mhz.append(float(parts[1]))
                maxes.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() in ("active", "1", "yes"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(mhz)) if mhz else None,
                "sm_max_mhz": float(max(maxes)) if maxes else None,
                "reasons": sorted(reasons), "samples": len(mhz)}


# ---------------------------------------------------------------- workload ---

def build_solvers(cb, precision: int = 0):
    mesh = cb.cgrid(WORKLOAD["designation"], **{k: v for k, v in WORKLOAD.items() if k != "designation"})
    settings = cb.Settings.defaults(inflow_intensity=INTENSITY, inflow_viscosity_ratio=VISCOSITY_RATIO,
                                    precision=precision)
    solvers = []
    for alpha in ALPHAS:
        s = cb.SimpleSolver.create(mesh, cb.freestream_conditions(mesh, 1.0, alpha), settings)
        s.set_turbulence_model(cb.MODEL_SST)
        s.initialise(*cb.uniform_field(mesh, 1.0, alpha, 1.0, REYNOLDS))
        solvers.append(s)
    return mesh, solvers


def converge_both_forms(cb, tolerance: float = 1e-6, cap: int = 6000) -> dict:
    """The benchmark pair solved to convergence in each form from the uniform
    start, batched (both solves in one launch per chunk, each stopping on its
    own): solves/min, iterations, and the mixed answers' differences from
    the FP64 ones (Cl, Cd, Cm, and Cp at every station)."""
    import torch
    out = {"tolerance": tolerance, "cap": cap}
    answers = {}
    for name, precision in (("plain", 0), ("mixed", 1)):
        mesh, solvers = build_solvers(cb, precision)
        batch = cb.Batch(solvers)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        taken, _ = batch.iterate(cap, tolerance)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        forces = [s.forces(1.0, a, 1.0) for s, a in zip(solvers, ALPHAS)]
        answers[name] = forces
        out[name] = {"solves_per_min": 60.0 * len(solvers) / wall, "wall_s": wall,
                     "iterations": list(taken),
                     "cl": [f[0].lift_coefficient for f in forces],
                     "cd": [f[0].drag_coefficient for f in forces]}
        batch.close()
        for s in solvers:
            s.close()
    p, m = answers["plain"], answers["mixed"]
    out["mixed_vs_plain"] = {
        "solves_per_min_ratio": out["mixed"]["solves_per_min"] / out["plain"]["solves_per_min"],
        "dcl": [abs(b[0].lift_coefficient - a[0].lift_coefficient) for a, b in zip(p, m)],
        "dcd": [abs(b[0].drag_coefficient - a[0].drag_coefficient) for a, b in zip(p, m)],
        "dcm": [abs(b[0].moment_coefficient - a[0].moment_coefficient) for a, b in zip(p, m)],
        "dcp_inf": [float(np.max(np.abs(b[1] - a[1]))) for a, b in zip(p, m)]}
    return out


def measured_peak() -> tuple[float, str]:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def committed_traffic(name: str = "simple_kernel_c2_sst_fp64.md") -> float | None:
    """DRAM bytes per launch of simpleKernel on this workload, from the
    committed ncu summary (its `traffic_bytes_per_launch:` line)."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":", 1)[1])
    except (OSError, ValueError):
        pass
    return None


# ------------------------------------------------------------- CPU leg ---

def _ref_worker(args):
    """One process: the reference solver (or the oracle port) on one solve,
    `warm` untimed then `count` timed iterations. Returns (cells, seconds, kind)."""
    alpha, warm, count = args
    sys.path.insert(0, ROOT)
    sys.path.insert(0, PKG)
    from oracle import reference as R
    w = WORKLOAD
    settings = np.array([0.5, 0.2, 3, 200, 0.01, 0, 0.5, INTENSITY, VISCOSITY_RATIO, 0.0, 1, 1.0])
    if R.available():
        m = R.RefMesh.cgrid(w["designation"], w["surface_points"], w["wake_points"],
                            w["normal_points"], w["first_layer_height"], w["upstream_chords"],
                            w["downstream_chords"], w["vertical_chords"])
        kind, vel, pres = m.conditions(1.0, alpha, 1.0, REYNOLDS)
        s = R.RefSolver(m, kind, vel, pres, settings, turbulence=2)
        s.initialise(*m.uniform(1.0, alpha, 1.0, REYNOLDS))
        label = "reference"
    else:
        import cfd_b200 as cb
        from oracle import port
        m = cb.cgrid(w["designation"], **{k: v for k, v in w.items() if k != "designation"})
        s = port.OracleSolver(m, cb.freestream_conditions(m, 1.0, alpha), settings, 2,
                              port.LEXICOGRAPHIC)
        s.initialise(*cb.uniform_field(m, 1.0, alpha, 1.0, REYNOLDS))
        label = "port"
    s.iterate(warm)
    t0 = time.perf_counter()
    s.iterate(count)
    return m.cells, time.perf_counter() - t0, label


def cpu_baseline(iterations: int = 60) -> dict:
    """The reference CPU solver on one core: a bounded sample of the workload
    (one of its solves, `iterations` outer iterations after 3 warm-up)."""
    cells, seconds, kind = _ref_worker((ALPHAS[-1], 3, iterations))
    return {"value": cells * iterations / seconds, "unit": UNIT, "cores": 1, "kind": kind,
            "sample": f"{iterations} SIMPLE iterations of one 384x96 SST solve (alpha {ALPHAS[-1]}), "
                      f"single thread, {seconds:.1f} s"}


def run_reference_arm(args) -> None:
    import multiprocessing as mp
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    procs = max(1, min(cores, 64))
    per_step = 1
    count = max(1, args.steps) * per_step
    jobs = [(ALPHAS[k % len(ALPHAS)], args.warmup, count) for k in range(procs)]
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        results = pool.map(_ref_worker, jobs)
    wall = time.perf_counter() - t0
    cells = sum(r[0] for r in results)
    slowest = max(r[1] for r in results)
    value = cells * count / slowest
    kind = results[0][2]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": slowest / count * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": config({"processes": procs}),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": kind,
                         "sample": f"{procs} independent solves (alpha {ALPHAS}) x {count} timed "
                                   f"iterations after {args.warmup} warm-up, one process per core; "
                                   f"wall {wall:.1f} s"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------- GPU arm ---

def run_ours(args) -> None:
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)

    import cfd_b200 as cb
    cb.set_device(torch.cuda.current_device())
    mixed = args.form == "mixed"
    mesh, solvers = build_solvers(cb, 1 if mixed else 0)
    batch = cb.Batch(solvers)
    cells = mesh.cells * len(solvers)
    # A stream of our own: events, the L2 flush and the solver launches all go
    # on it (torch's default stream is the legacy NULL stream, handle 0).
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    handle = stream.cuda_stream
    assert handle != 0
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    # warm-up (untimed), also moves the flow off its uniform start
    launch = batch.graph_launch if args.graph else batch.launch
    for _ in range(args.warmup):
        flush.zero_()
        launch(1, handle)
    torch.cuda.synchronize()

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(torch.cuda.current_device()) as clocks:
        for k in range(args.steps):
            flush.zero_()
            starts[k].record(stream)
            launch(1, handle)
            ends[k].record(stream)
        torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    step_ms = np.array([s.elapsed_time(e) for s, e in zip(starts, ends)])
    total_s = float(step_ms.sum()) / 1e3
    gpu_launches = args.steps
    _, monitors = batch.monitors()
    finite = all(math.isfinite(m.continuity) for m in monitors)

    # mean executed CG iterations: 20 more iterations with history
    cg = []
    for s in solvers:
        _, hist = s.iterate(20, history=True)
        cg.extend(hist[:, 5].tolist())
    mean_cg = float(np.mean(cg))

    # e2e through the C ABI from pinned host buffers
    e2e_steps = max(5, min(50, args.steps))
    states = []
    for s in solvers:
        arrays = {}
        for name in ("U", "V", "P", "K", "OMEGA", "MUT", "MU_EFF"):
            t = torch.empty(mesh.cells, dtype=torch.float64, pin_memory=True)
            t.numpy()[:] = s.read(name)
            arrays[name] = t
        t = torch.empty(mesh.faces, dtype=torch.float64, pin_memory=True)
        t.numpy()[:] = s.read("MASS_FLUX")
        arrays["MASS_FLUX"] = t
        states.append(arrays)
    h2d = sum(sum(t.numel() * 8 for t in a.values()) for a in states)
    d2h = len(solvers) * 136
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        for s, a in zip(solvers, states):
            s.load_state(u=a["U"].numpy(), v=a["V"].numpy(), p=a["P"].numpy(),
                         mass_flux=a["MASS_FLUX"].numpy(), k=a["K"].numpy(),
                         omega=a["OMEGA"].numpy(), mut=a["MUT"].numpy(), mu_eff=a["MU_EFF"].numpy())
        taken, mons = batch.iterate(1)
        assert all(t == 1 for t in taken)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0

    # multi-rank: max time over ranks, cells summed
    if dist is not None:
        (total_s, e2e_s), all_cells = reduce_over_ranks([total_s, e2e_s], cells, dist, "cuda")
    else:
        all_cells = float(cells)
    value = all_cells * args.steps / total_s
    e2e_value = all_cells * e2e_steps / e2e_s

    if rank == 0:
        import bytes_model
        peak, peak_kind = measured_peak()
        if mixed:
            per_launch_bytes = bytes_model.bytes_per_cell_iteration_mixed(True, mean_cg) * cells
        else:
            per_launch_bytes = bytes_model.bytes_per_cell_iteration(True, mean_cg) * cells
        mean_launch_s = float(np.mean(step_ms)) / 1e3
        achieved = per_launch_bytes / mean_launch_s / 1e9
        traffic = committed_traffic("simple_kernel_c2_sst_mixed.md" if mixed else "simple_kernel_c2_sst_fp64.md")
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs",
                    "traffic": traffic,
                    "kernel": "simpleKernel", "bytes_per_launch_algorithmic": per_launch_bytes,
                    "mean_cg_iterations": mean_cg}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": float(np.mean(step_ms)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32/f64" if mixed else "f64",
            "data": "synthetic",
            "config": config({"cluster_shape": list(batch.shape()), "launch": "cuda graph" if args.graph else "direct"}
                             if not mixed else
                             {"cluster_shape": list(batch.shape()),
                              "workload": "NACA0012 k-omega SST Re1e6 C-grid 384x96 (medium), alpha 0 "
                                          "and 4 deg, mixed FP32/FP64 form, batched in one launch",
                              "precision": "mixed: FP64 assembly/state, FP32 sweeps and multigrid CG"}),
            "roofline": roofline,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": gpu_launches, "clocks": clocks.summary(),
            "finite": finite,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline()
        if world == 1 and not args.no_convergence:
            line["convergence"] = converge_both_forms(cb)
        print(json.dumps(line), flush=True)
    batch.close()
    for s in solvers:
        s.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def reduce_over_ranks(times, cells, dist, device):
    """Replicas: the job's times are the slowest rank's, its work the sum of
    every rank's. Every rank calls this with the same number of values."""
    import torch
    t = torch.tensor([float(x) for x in times], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor([float(cells)], dtype=torch.float64, device=device)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return [float(x) for x in t.tolist()], float(c.item())


# ------------------------------------------------- engine workloads ---

GRIDS = {  # (surface, wake, normal) points; cells 192x48, 384x96, 768x192
    "coarse": (64, 33, 49), "medium": (128, 65, 97), "fine": (256, 129, 193),
}


def _percentiles(values):
    if not values:
        return {"p50": None, "p95": None, "p99": None}
    a = np.sort(np.asarray(values))
    return {f"p{q}": float(np.percentile(a, q)) for q in (50, 95, 99)}


def _summarise(results, wall_s, cb):
    statuses = {}
    for r in results:
        statuses[cb.STATUS_NAMES[r.status]] = statuses.get(cb.STATUS_NAMES[r.status], 0) + 1
    cell_iters = float(sum(r.cells * r.iterations for r in results))
    lat = [r.finished_s - r.submitted_s for r in results]
    return {"solves": len(results), "wall_s": wall_s, "solves_per_min": 60.0 * len(results) / wall_s,
            "cell_iters_per_s": cell_iters / wall_s, "statuses": statuses,
            "time_to_convergence_s": _percentiles(lat),
            "iterations": _percentiles([r.iterations for r in results])}


def _polar_requests(cb, args, precision):
    settings = cb.Settings.defaults(inflow_viscosity_ratio=VISCOSITY_RATIO, precision=precision)
    reqs = []
    for alpha in range(-4, 17):
        s, w, n = GRIDS["fine"]
        reqs.append(cb.request("2412", float(alpha), 3e6, tolerance=args.tolerance,
                               max_iterations=args.cap, surface_points=s, wake_points=w,
                               normal_points=n, first_layer_height=5e-6, settings=settings))
    for level, fl in (("coarse", 2e-3), ("medium", 1e-5), ("fine", 5e-6)):
        s, w, n = GRIDS[level]
        reqs.append(cb.request("0012", 4.0, 1e6, tolerance=args.tolerance, max_iterations=args.cap,
                               surface_points=s, wake_points=w, normal_points=n,
                               first_layer_height=fl, settings=settings))
    return reqs


def run_polar(args) -> None:
    """21-point NACA 2412 SST Re 3e6 polar (alpha -4..16 step 1) on
    the fine 768x192 C-grid, plus NACA 0012 SST Re 1e6 alpha 4 on the coarse,
    medium and fine grids, all resident at once in one engine; run in the
    plain FP64 form and in the mixed FP32/FP64 form, with the mixed answers'
    differences from the FP64 ones (Cl, Cd, Cm, and Cp at every station)."""
    import torch
    torch.cuda.set_device(0)
    import cfd_b200 as cb
    cb.set_device(0)
    forms = ("plain", "mixed") if args.precision == "both" else (args.precision,)
    out = {"workload": "polar: NACA2412 SST Re3e6 768x192 alpha -4..16 + NACA0012 SST Re1e6 "
                       "alpha 4 on 192x48/384x96/768x192", "tolerance": args.tolerance,
           "cap": args.cap, "chunk": args.chunk}
    runs = {}
    for form in forms:
        reqs = _polar_requests(cb, args, 0 if form == "plain" else 1)
        engine = cb.Engine(chunk=args.chunk)
        t0 = time.perf_counter()
        results = sorted(engine.run(reqs), key=lambda r: r.id)
        wall = time.perf_counter() - t0
        cps = {r.id: engine.surface(r.id) for r in results if r.status != 2}
        engine.close()
        runs[form] = (results, cps)
        summary = _summarise(results, wall, cb)
        if args.csv:
            sweep = [r for r in results if reqs[r.id].designation.decode() == "2412"]
            with open(f"{args.csv}_{form}.csv", "w") as fh:
                fh.write(cb.polar_csv(sweep, [reqs[r.id].alpha_deg for r in sweep], "NACA 2412",
                                      "768x192", 3e6, 1.0))
        summary["polar"] = [{"alpha": reqs[r.id].alpha_deg, "section": reqs[r.id].designation.decode(),
                             "cells": r.cells, "status": cb.STATUS_NAMES[r.status],
                             "iterations": r.iterations, "ctas": r.cluster_size,
                             "cl": r.lift_coefficient,
                             "cd": r.drag_coefficient, "cm": r.moment_coefficient,
                             "continuity": r.continuity} for r in results]
        out[form] = summary
    if len(forms) == 2:
        (rp, cpp), (rm, cpm) = runs["plain"], runs["mixed"]
        rows = []
        for a, b in zip(rp, rm):
            row = {"id": a.id, "dcl": abs(b.lift_coefficient - a.lift_coefficient),
                   "dcd": abs(b.drag_coefficient - a.drag_coefficient),
                   "dcm": abs(b.moment_coefficient - a.moment_coefficient),
                   "iterations_plain": a.iterations, "iterations_mixed": b.iterations}
            if a.id in cpp and b.id in cpm and len(cpp[a.id]) == len(cpm[b.id]):
                row["dcp_inf"] = float(np.max(np.abs(cpm[b.id] - cpp[a.id])))
            rows.append(row)
        both_converged = [r for r, a, b in zip(rows, rp, rm) if a.status == 0 and b.status == 0]
        out["mixed_vs_plain"] = {
            "solves_per_min_ratio": out["mixed"]["solves_per_min"] / out["plain"]["solves_per_min"],
            "max_dcl": max(r["dcl"] for r in rows), "max_dcd": max(r["dcd"] for r in rows),
            "max_dcm": max(r["dcm"] for r in rows),
            "max_dcp_inf": max((r.get("dcp_inf", 0.0) for r in rows), default=None),
            "max_dcl_both_converged": max((r["dcl"] for r in both_converged), default=None),
            "per_solve": rows}
    print(json.dumps(out), flush=True)


def run_settled(args) -> None:
    """Accuracy of the mixed form where it can be judged: NACA 0012 SST Re 1e6
    alpha 0 and 4 on 384x96 and NACA 2412 SST Re 3e6 alpha 2 on 768x192, each
    solved in both forms to worst residual 1e-8 (or 12,000 iterations), when
    Cl has settled to ~1e-5; at the production tolerance 1e-6 neither form's
    Cl has (it still moves by ~1e-2), so differences there measure
    convergence, not precision."""
    import torch
    torch.cuda.set_device(0)
    import cfd_b200 as cb
    cb.set_device(0)
    tol, cap = 1e-8, 12000
    cases = [("0012", 0.0, 1e6, "medium", 1e-5), ("0012", 4.0, 1e6, "medium", 1e-5),
             ("2412", 2.0, 3e6, "fine", 5e-6)]
    out = {"workload": "settled: NACA0012 SST Re1e6 384x96 alpha 0/4, NACA2412 SST Re3e6 768x192 alpha 2",
           "tolerance": tol, "cap": cap}
    answers = {}
    for form, precision in (("plain", 0), ("mixed", 1)):
        settings = cb.Settings.defaults(inflow_viscosity_ratio=VISCOSITY_RATIO, precision=precision)
        reqs = []
        for des, alpha, re, level, fl in cases:
            sp, wk, nm = GRIDS[level]
            reqs.append(cb.request(des, alpha, re, tolerance=tol, max_iterations=cap, surface_points=sp,
                                   wake_points=wk, normal_points=nm, first_layer_height=fl,
                                   settings=settings))
        engine = cb.Engine(chunk=args.chunk)
        t0 = time.perf_counter()
        results = sorted(engine.run(reqs), key=lambda r: r.id)
        wall = time.perf_counter() - t0
        cps = {r.id: engine.surface(r.id) for r in results if r.status != 2}
        engine.close()
        answers[form] = (results, cps)
        out[form] = {"wall_s": wall, "per_solve": [
            {"case": f"{c[0]} alpha {c[1]:g} {c[3]}", "status": cb.STATUS_NAMES[r.status],
             "iterations": r.iterations, "cl": r.lift_coefficient, "cd": r.drag_coefficient,
             "cm": r.moment_coefficient} for c, r in zip(cases, results)]}
    (rp, cpp), (rm, cpm) = answers["plain"], answers["mixed"]
    out["mixed_vs_plain"] = [
        {"case": f"{c[0]} alpha {c[1]:g} {c[3]}",
         "dcl": abs(b.lift_coefficient - a.lift_coefficient),
         "dcd": abs(b.drag_coefficient - a.drag_coefficient),
         "dcm": abs(b.moment_coefficient - a.moment_coefficient),
         "dcp_inf": (float(np.max(np.abs(cpm[b.id] - cpp[a.id])))
                     if a.id in cpp and b.id in cpm and len(cpp[a.id]) == len(cpm[b.id]) else None)}
        for c, a, b in zip(cases, rp, rm)]
    print(json.dumps(out), flush=True)


def serving_stream(n: int, rate: float, seed: int):
    """seeded Poisson arrivals of NACA 4-digit SST requests."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    out = []
    for k in range(n):
        m = int(rng.integers(0, 7))
        pos = int(rng.integers(2, 7)) if m > 0 else 0
        thick = int(rng.integers(6, 22))
        alpha = float(rng.uniform(-5.0, 15.0))
        re = float(10 ** rng.uniform(5.0, 7.0))
        level = rng.choice(["coarse", "medium", "fine"], p=[0.5, 0.35, 0.15])
        out.append((float(t[k]), f"{m}{pos}{thick:02d}", alpha, re, str(level),
                    2.5e-5 * (1e6 / re) ** 0.9))
    return out


def run_serve(args) -> None:
    import torch
    torch.cuda.set_device(0)
    import cfd_b200 as cb
    cb.set_device(0)
    stream = serving_stream(args.requests, args.rate, args.seed)
    settings = cb.Settings.defaults(inflow_viscosity_ratio=VISCOSITY_RATIO,
                                    precision=1 if args.precision == "mixed" else 0)
    engine = cb.Engine(chunk=args.chunk, tuned=True)  # a saturated GPU: the occupancy tuner
    t0 = engine.clock()
    submitted, results = 0, []
    wall0 = time.perf_counter()
    while len(results) < len(stream):
        now = engine.clock() - t0
        while submitted < len(stream) and stream[submitted][0] <= now:
            _, des, alpha, re, level, fl = stream[submitted]
            s, w, n = GRIDS[level]
            engine.submit(cb.request(des, alpha, re, tolerance=args.tolerance,
                                     max_iterations=args.cap, surface_points=s, wake_points=w,
                                     normal_points=n, first_layer_height=fl, settings=settings))
            submitted += 1
        active, queued = engine.step()
        results.extend(engine.results())
        if active == 0 and queued == 0 and submitted < len(stream):
            time.sleep(max(0.0, min(0.05, stream[submitted][0] - (engine.clock() - t0))))
    wall = time.perf_counter() - wall0
    out = _summarise(results, wall, cb)
    out.update({"workload": f"serve: Poisson lambda={args.rate}/s, {args.requests} NACA 4-digit SST "
                            f"requests (seed {args.seed}), meshes 192x48/384x96/768x192 at "
                            "0.5/0.35/0.15", "precision": args.precision if args.precision == "mixed" else "plain",
                "tolerance": args.tolerance, "cap": args.cap,
                "chunk": args.chunk})
    print(json.dumps(out), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-convergence", action="store_true",
                    help="skip solving the pair to convergence in both forms")
    ap.add_argument("--workload", choices=("c2", "polar", "serve", "settled"), default="c2",
                    help="c2: the benchmark line (default); polar / serve / settled: engine workloads")
    ap.add_argument("--tolerance", type=float, default=1e-6)
    ap.add_argument("--cap", type=int, default=4000)
    ap.add_argument("--chunk", type=int, default=32)
    ap.add_argument("--requests", type=int, default=512)
    ap.add_argument("--rate", type=float, default=4.0)
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--csv", default="",
                    help="polar: write the 2412 sweep of each form as <prefix>_<form>.csv "
                         "in the reference's polar CSV layout")
    ap.add_argument("--graph", action="store_true",
                    help="c2: replay each step's launch from a CUDA graph")
    ap.add_argument("--form", choices=("plain", "mixed"), default="plain",
                    help="c2: the form the benchmark line times (plain FP64 by default)")
    ap.add_argument("--precision", choices=("plain", "mixed", "both"), default="both",
                    help="polar: which form(s) to run; serve: plain unless 'mixed'")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be at least 3")
    if args.workload == "polar":
        run_polar(args)
    elif args.workload == "settled":
        run_settled(args)
    elif args.workload == "serve":
        run_serve(args)
    elif args.impl == "reference":
        run_reference_arm(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
