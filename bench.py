"""Benchmark: the batched polar of steady SIMPLE solves (k-omega SST, plain FP64).

Workload (one "step" = one SIMPLE outer iteration of every solve in it, all
in one batched launch, one thread-block cluster per solve):
  a 21-point NACA 2412 polar, Re 3e6, alpha -4..16 deg step 1, on the fine
  C-grid 768 x 192 cells (surface 256, wake 129, normal 193 points; first
  layer 5e-6 chord), plus NACA 0012 at Re 1e6, alpha 4 deg, on the coarse
  192 x 48 (first layer 2e-3), medium 384 x 96 (1e-5) and fine 768 x 192
  (5e-6) C-grids: 24 solves of uneven size, 3,290,112 cells resident at once
  (3.2 GB of device state). k-omega SST, inflow intensity 0.1 %, mu_t/mu 10;
  domains 10 chords upstream and vertically, 15 downstream. Synthetic inputs:
  the uniform freestream start of FlowField::uniform, advanced by the warm-up
  steps; no dataset exists for this path.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0). `value` is cell-iterations/s of the plain FP64
form over all ranks, timed with CUDA events around each step's launch on the
launching stream; the state (3.2 GB) is larger than the L2 (126 MB), and a
256 MiB buffer is written between timed steps besides. `e2e` is the same
metric through the C ABI from pinned host buffers: every step loads each
solve's state host->device, iterates the batch once and reads each solve's
u, v and p back. The same line carries the mixed FP32/FP64 form's figures on
the same workload, both forms' polar solved to convergence (solves/min,
time-to-convergence percentiles, per-point Cl/Cd/Cm/Cp differences) and the
reference's CPU solver timed on the host's cores. `--impl reference` times the
reference's own CPU solver (compiled from its sources into oracle/_ref) on the
same workload with the host's cores. Multi-GPU (torchrun): independent
replicas, one per GPU; no collective on the data path (weak scaling).
"""
from __future__ import annotations

import argparse
import contextlib
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
REYNOLDS = 1e6
INTENSITY = 0.001
VISCOSITY_RATIO = 10.0
EXTENTS = dict(upstream_chords=10.0, downstream_chords=15.0, vertical_chords=10.0)
GRIDS = {  # (surface, wake, normal) points; cells 192x48, 384x96, 768x192
    "coarse": (64, 33, 49), "medium": (128, 65, 97), "fine": (256, 129, 193),
}
# The batched polar: (designation, alpha, Reynolds, grid, first layer height)
POLAR = ([("2412", float(a), 3e6, "fine", 5e-6) for a in range(-4, 17)]
         + [("0012", 4.0, 1e6, "coarse", 2e-3), ("0012", 4.0, 1e6, "medium", 1e-5),
            ("0012", 4.0, 1e6, "fine", 5e-6)])
POLAR_NAME = ("batched polar: NACA2412 k-omega SST Re3e6 C-grid 768x192, alpha -4..16 step 1 "
              "(21 solves) + NACA0012 k-omega SST Re1e6 alpha 4 on 192x48/384x96/768x192, "
              "24 solves in one batch (one launch per cluster size)")
# The mixed form runs on clusters of at most 8 CTAs (the engine's default
# policy for it: smaller clusters fit more of its solves on the GPU).
MIXED_CLUSTER = 8
# The former headline pair (384 x 96, alpha 0 and 4), kept as --workload c2.
C2_ALPHAS = (0.0, 4.0)


def polar_config(extra=None):
    c = {"workload": POLAR_NAME, "solves": len(POLAR),
         "cells": sum(_cells(level) for _, _, _, level, _ in POLAR), "model": "k-omega SST",
         "precision": "fp64 plain (reference-parity form)",
         "l2": "state 3.2 GB > L2; a 256 MiB buffer is also written between timed steps",
         "parallelism": "replicas"}
    if extra:
        c.update(extra)
    return c


def _cells(level: str) -> int:
    s, w, n = GRIDS[level]
    return (2 * w + 2 * s - 2) * (n - 1)  # cellsI = 2 wake + 2 surface - 2


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

def _mesh(cb, designation, level, first_layer, cache):
    key = (designation, level, first_layer)
    if key not in cache:
        sp, wp, npn = GRIDS[level]
        cache[key] = cb.cgrid(designation, surface_points=sp, wake_points=wp, normal_points=npn,
                              first_layer_height=first_layer, **EXTENTS)
    return cache[key]


@contextlib.contextmanager
def _cluster_env(cluster: int):
    """CFD_CLUSTER_SIZE set to `cluster` for the solves created inside."""
    previous = os.environ.get("CFD_CLUSTER_SIZE")
    os.environ["CFD_CLUSTER_SIZE"] = str(cluster)
    try:
        yield
    finally:
        if previous is None:
            os.environ.pop("CFD_CLUSTER_SIZE", None)
        else:
            os.environ["CFD_CLUSTER_SIZE"] = previous


def plain_cluster(designation: str, level: str) -> int:
    """CTAs per solve of the plain form's batched polar. The 21 NACA 2412
    points take 16-CTA clusters: a B200 holds 7 of those at once, so they fill
    exactly three waves. The NACA 0012 trio runs beside them on the SMs those
    clusters leave free, in a launch of its own: 768x192 on 8 CTAs, the two
    smaller grids on 4. (All 24 on 16 CTAs take a fourth wave for the one
    768x192 0012 solve: 18.9 against 17.9 ms per step.)"""
    if designation == "2412":
        return 16
    return 8 if level == "fine" else 4


def polar_solvers(cb, precision: int = 0, cluster: int | None = None, count: int | None = None):
    """The 24 solves of the batched polar (or its first `count`, for a
    profiling capture of a smaller case), created on the device from the
    uniform start. `cluster` fixes the CTAs per solve (the library's
    CFD_CLUSTER_SIZE knob), else each solve takes `plain_cluster`'s."""
    settings = cb.Settings.defaults(inflow_intensity=INTENSITY, inflow_viscosity_ratio=VISCOSITY_RATIO,
                                    precision=precision)
    meshes, solvers = {}, []
    for des, alpha, re, level, fl in POLAR[:count]:
        mesh = _mesh(cb, des, level, fl, meshes)
        with _cluster_env(cluster if cluster is not None else plain_cluster(des, level)):
            s = cb.SimpleSolver.create(mesh, cb.freestream_conditions(mesh, 1.0, alpha), settings)
        s.set_turbulence_model(cb.MODEL_SST)
        s.initialise(*cb.uniform_field(mesh, 1.0, alpha, 1.0, re))
        solvers.append(s)
    return solvers


def c2_solvers(cb, precision: int = 0):
    """The 384x96 NACA 0012 pair (alpha 0 and 4) of --workload c2."""
    mesh = _mesh(cb, "0012", "medium", 1e-5, {})
    settings = cb.Settings.defaults(inflow_intensity=INTENSITY, inflow_viscosity_ratio=VISCOSITY_RATIO,
                                    precision=precision)
    out = []
    for alpha in C2_ALPHAS:
        s = cb.SimpleSolver.create(mesh, cb.freestream_conditions(mesh, 1.0, alpha), settings)
        s.set_turbulence_model(cb.MODEL_SST)
        s.initialise(*cb.uniform_field(mesh, 1.0, alpha, 1.0, REYNOLDS))
        out.append(s)
    return out


def measured_peak() -> tuple[float, str]:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def committed_traffic(name: str) -> float | None:
    """DRAM bytes per launch of simpleKernel on a workload, from a committed
    ncu summary (its `traffic_bytes_per_launch:` line)."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":", 1)[1])
    except (OSError, ValueError):
        pass
    return None


def algorithmic_bytes(solvers, cg_iterations, mixed: bool) -> float:
    """Bytes one batched launch of one iteration must move (bytes_model), summed
    over the solves with each solve's executed CG (or inner multigrid-CG)
    iterations."""
    import bytes_model
    total = 0.0
    for s, n in zip(solvers, cg_iterations):
        per = (bytes_model.bytes_per_cell_iteration_mixed(True, n) if mixed
               else bytes_model.bytes_per_cell_iteration(True, n))
        total += per * s.mesh.cells
    return total


# ------------------------------------------------------------- CPU leg ---

def _ref_worker(args):
    """One process: the reference solver (or, where it was not built, the
    oracle port) on a list of solves: `warm` untimed, then `count` timed
    iterations of every solve, round-robin like one batched step after
    another. Returns (cells, seconds, kind)."""
    solves, warm, count = args
    sys.path.insert(0, ROOT)
    sys.path.insert(0, PKG)
    from oracle import reference as R
    settings = np.array([0.5, 0.2, 3, 200, 0.01, 0, 0.5, INTENSITY, VISCOSITY_RATIO, 0.0, 1, 1.0])
    built = []
    for des, alpha, re, level, fl in solves:
        sp, wp, npn = GRIDS[level]
        if R.available():
            m = R.RefMesh.cgrid(des, sp, wp, npn, fl, EXTENTS["upstream_chords"],
                                EXTENTS["downstream_chords"], EXTENTS["vertical_chords"])
            kind, vel, pres = m.conditions(1.0, alpha, 1.0, re)
            s = R.RefSolver(m, kind, vel, pres, settings, turbulence=2)
            s.initialise(*m.uniform(1.0, alpha, 1.0, re))
            label = "reference"
        else:
            import cfd_b200 as cb
            from oracle import port
            m = cb.cgrid(des, surface_points=sp, wake_points=wp, normal_points=npn,
                         first_layer_height=fl, **EXTENTS)
            s = port.OracleSolver(m, cb.freestream_conditions(m, 1.0, alpha), settings, 2,
                                  port.LEXICOGRAPHIC)
            s.initialise(*cb.uniform_field(m, 1.0, alpha, 1.0, re))
            label = "port"
        built.append((m, s))
    for _ in range(warm):
        for _, s in built:
            s.iterate(1)
    t0 = time.perf_counter()
    for _ in range(count):
        for _, s in built:
            s.iterate(1)
    return sum(m.cells for m, _ in built), time.perf_counter() - t0, label


def _processes(work: int) -> int:
    return max(1, min(os.cpu_count() or 1, work))


def cpu_baseline(iterations: int = 10) -> dict:
    """The reference CPU solver on the host's cores: a bounded sample of the
    workload, one fine-grid solve of the polar per process (768x192 NACA 2412,
    a different incidence in each), 2 untimed then `iterations` timed outer
    iterations; the aggregate rate is every process's cells x iterations over
    the slowest process's time."""
    import multiprocessing as mp
    fine = [p for p in POLAR if p[3] == "fine"]
    procs = _processes(len(fine))
    jobs = [([fine[k]], 2, iterations) for k in range(procs)]
    with mp.get_context("spawn").Pool(procs) as pool:
        results = pool.map(_ref_worker, jobs)
    cells = sum(r[0] for r in results)
    slowest = max(r[1] for r in results)
    return {"value": cells * iterations / slowest, "unit": UNIT, "cores": procs, "kind": results[0][2],
            "sample": f"{procs} processes, one 768x192 NACA 2412 SST solve each (alpha "
                      f"{fine[0][1]:g}..{fine[procs - 1][1]:g}), {iterations} timed iterations after 2, "
                      f"slowest {slowest:.1f} s"}


def run_reference_arm(args) -> None:
    """The reference's CPU solver on the same 24-solve workload: the solves
    are dealt round-robin to one process per host core (at most one per
    solve); a step is one outer iteration of every solve."""
    import multiprocessing as mp
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    workload = POLAR if args.workload != "c2" else [("0012", a, REYNOLDS, "medium", 1e-5) for a in C2_ALPHAS]
    procs = _processes(len(workload))
    count = max(1, args.steps)
    jobs = [([workload[k] for k in range(p, len(workload), procs)], args.warmup, count)
            for p in range(procs)]
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(procs) as pool:
        results = pool.map(_ref_worker, jobs)
    wall = time.perf_counter() - t0
    cells = sum(r[0] for r in results)
    slowest = max(r[1] for r in results)
    value = cells * count / slowest
    kind = results[0][2]
    config = polar_config({"processes": procs}) if args.workload != "c2" else c2_config({"processes": procs})
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": slowest / count * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": config,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": kind,
                         "sample": f"{len(workload)} solves over {procs} processes (one per core), "
                                   f"{count} timed steps after {args.warmup} warm-up, each step one "
                                   f"iteration of every solve; wall {wall:.1f} s"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def c2_config(extra=None):
    c = {"workload": "NACA0012 k-omega SST Re1e6 C-grid 384x96 (medium), alpha 0 and 4 deg, "
                     "plain FP64, batched in one launch",
         "cells_per_solve": 384 * 96, "solves": len(C2_ALPHAS), "model": "k-omega SST",
         "precision": "fp64 plain (reference-parity form)",
         "l2": "flushed between timed steps (256 MiB write)", "parallelism": "replicas"}
    if extra:
        c.update(extra)
    return c


# ------------------------------------------------------------- GPU arm ---

def _timed_steps(torch, batch, handle, stream, flush, steps, warmup, dist, launch=None):
    """W untimed then K timed one-iteration launches of a batch, each bracketed
    by CUDA events on the launching stream, the L2 flush between them."""
    launch = launch or batch.launch
    for _ in range(warmup):
        flush.zero_()
        launch(1, handle)
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(torch.cuda.current_device()) as clocks:
        for k in range(steps):
            flush.zero_()
            starts[k].record(stream)
            launch(1, handle)
            ends[k].record(stream)
        torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    return np.array([a.elapsed_time(b) for a, b in zip(starts, ends)]), clocks.summary()


def _e2e(torch, batch, solvers, steps, dist):
    """The metric through the C ABI with host buffers: every step loads each
    solve's state from pinned host memory, iterates the batch once, and reads
    each solve's u, v and p back into pinned host memory. Returns (seconds,
    h2d bytes per step, d2h bytes per step)."""
    def pinned(n):
        return torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()

    states, outs = [], []
    for s in solvers:
        a = {}
        for name in ("U", "V", "P", "K", "OMEGA", "MUT", "MU_EFF", "MASS_FLUX"):
            buf = pinned(s.mesh.faces if name == "MASS_FLUX" else s.mesh.cells)
            s.read_into(name, buf)
            a[name] = buf
        states.append(a)
        outs.append({name: pinned(s.mesh.cells) for name in ("U", "V", "P")})
    h2d = sum(sum(b.nbytes for b in a.values()) for a in states)
    d2h = sum(sum(b.nbytes for b in o.values()) for o in outs) + len(solvers) * 136
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(steps):
        for s, a in zip(solvers, states):
            s.load_state(u=a["U"], v=a["V"], p=a["P"], mass_flux=a["MASS_FLUX"], k=a["K"],
                         omega=a["OMEGA"], mut=a["MUT"], mu_eff=a["MU_EFF"])
        taken, _ = batch.iterate(1)
        assert all(t == 1 for t in taken)
        for s, o in zip(solvers, outs):
            for name, buf in o.items():
                s.read_into(name, buf)
    torch.cuda.synchronize()
    return time.perf_counter() - t0, h2d, d2h


def _roofline(solvers, cg, step_ms, mixed, profile):
    peak, peak_kind = measured_peak()
    per_launch = algorithmic_bytes(solvers, cg, mixed)
    achieved = per_launch / (float(np.mean(step_ms)) / 1e3) / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs",
            "traffic": committed_traffic(profile), "kernel": "simpleKernel",
            "bytes_per_launch_algorithmic": per_launch,
            "mean_cg_iterations": float(np.average(cg, weights=[s.mesh.cells for s in solvers]))}


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
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)

    import cfd_b200 as cb
    cb.set_device(torch.cuda.current_device())
    c2 = args.workload == "c2"
    mixed_only = args.form == "mixed"
    if c2:
        solvers = c2_solvers(cb, 1 if mixed_only else 0)
    else:
        solvers = polar_solvers(cb, 1 if mixed_only else 0, MIXED_CLUSTER if mixed_only else None,
                                args.solves)
    batch = cb.Batch(solvers)
    cells = sum(s.mesh.cells for s in solvers)
    # A stream of our own: events, the L2 flush and the solver launches all go
    # on it (torch's default stream is the legacy NULL stream, handle 0).
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    handle = stream.cuda_stream
    assert handle != 0
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    launch = batch.graph_launch if args.graph else batch.launch
    step_ms, clocks = _timed_steps(torch, batch, handle, stream, flush, args.steps, args.warmup, dist,
                                   launch)
    total_s = float(step_ms.sum()) / 1e3
    _, monitors = batch.monitors()
    finite = all(math.isfinite(m.continuity) for m in monitors)
    cg = [float(m.pressure_iterations) for m in monitors]  # executed in the last timed step
    shape = list(batch.shape())

    e2e_steps = max(3, min(10, args.steps))
    e2e_s, h2d, d2h = _e2e(torch, batch, solvers, e2e_steps, dist)

    # the mixed FP32/FP64 form on the same workload (its own batch)
    mixed = None
    if not mixed_only and not c2 and not args.no_mixed:
        batch.close()
        for s in solvers:
            s.close()
        m_solvers = polar_solvers(cb, 1, MIXED_CLUSTER, args.solves)
        m_batch = cb.Batch(m_solvers)
        m_ms, m_clocks = _timed_steps(torch, m_batch, handle, stream, flush, args.steps, args.warmup, dist)
        _, m_mon = m_batch.monitors()
        m_inner = [float(m.pressure_iterations) for m in m_mon]
        m_total = float(m_ms.sum()) / 1e3
        mixed = {"ms_per_step": float(np.mean(m_ms)), "total_s": m_total, "shape": list(m_batch.shape()),
                 "clocks": m_clocks, "inner": m_inner, "solvers": m_solvers,
                 "finite": all(math.isfinite(m.continuity) for m in m_mon)}
        m_batch.close()
    # multi-rank: max time over ranks, cells summed
    times = [total_s, e2e_s] + ([mixed["total_s"]] if mixed else [])
    if dist is not None:
        times, all_cells = reduce_over_ranks(times, cells, dist, "cuda")
    else:
        all_cells = float(cells)
    value = all_cells * args.steps / times[0]
    e2e_value = all_cells * e2e_steps / times[1]

    if rank == 0:
        profile = ("simple_kernel_c2_sst_mixed.md" if mixed_only else "simple_kernel_c2_sst_fp64.md") if c2 \
            else ("simple_kernel_polar_mixed.md" if mixed_only else "simple_kernel_polar_fp64.md")
        roofline = _roofline(solvers, cg, step_ms, mixed_only, profile)
        config = c2_config() if c2 else polar_config({"solves": len(solvers), "cells": cells})
        if not c2 and args.solves is not None:
            config["workload"] += f" (only the first {len(solvers)} solves: a profiling case)"
        config.update({"cluster_shape": shape, "cluster_sizes": sorted(
                           {plain_cluster(d, lv) for d, _, _, lv, _ in POLAR[:args.solves]}, reverse=True)
                       if not (c2 or mixed_only) else [shape[0]], "launch": "cuda graph" if args.graph else "direct",
                       "cg_iterations_per_solve": cg})
        if mixed_only:
            config["precision"] = "mixed: FP64 assembly/state, FP32 sweeps and multigrid CG"
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": float(np.mean(step_ms)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32/f64" if mixed_only else "f64", "data": "synthetic", "config": config,
            "roofline": roofline,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": args.steps * len(config["cluster_sizes"]), "clocks": clocks, "finite": finite,
        }
        if mixed is not None:
            m_value = all_cells * args.steps / times[2]
            line["mixed"] = {
                "value": m_value, "unit": UNIT, "ms_per_step": mixed["ms_per_step"],
                "vs_plain": m_value / value, "cluster_shape": mixed["shape"], "dtype": "f32/f64",
                "inner_iterations_per_solve": mixed["inner"], "clocks": mixed["clocks"],
                "finite": mixed["finite"],
                "roofline": _roofline(mixed["solvers"], mixed["inner"], np.array([mixed["ms_per_step"]]),
                                      True, "simple_kernel_polar_mixed.md")}
            for s in mixed["solvers"]:
                s.close()
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline()
        if world == 1 and not args.no_convergence and not c2:
            line["polar"] = polar_to_tolerance(cb, args.tolerance, args.cap, args.chunk)
            if "cpu_baseline" in line:
                line["polar"]["reference_cpu_estimate"] = reference_polar_estimate(
                    line["polar"]["plain"]["points"], line["cpu_baseline"])
        print(json.dumps(line), flush=True)
    if mixed is None:
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
            "queue_s": _percentiles([r.started_s - r.submitted_s for r in results]),
            "mesh_s": _percentiles([r.mesh_s for r in results if r.mesh_s > 0.0]),
            "iterations": _percentiles([r.iterations for r in results])}


def _polar_requests(cb, tolerance, cap, precision):
    settings = cb.Settings.defaults(inflow_intensity=INTENSITY, inflow_viscosity_ratio=VISCOSITY_RATIO,
                                    precision=precision)
    reqs = []
    for des, alpha, re, level, fl in POLAR:
        sp, wp, npn = GRIDS[level]
        reqs.append(cb.request(des, alpha, re, tolerance=tolerance, max_iterations=cap,
                               surface_points=sp, wake_points=wp, normal_points=npn,
                               first_layer_height=fl, settings=settings))
    return reqs


def reference_polar_estimate(points, cpu: dict) -> dict:
    """The reference's solves/min on the same polar, estimated rather than run
    (a run would take hours): the plain form's iteration counts per point
    (the reference's algorithm, which it follows to rounding) times the
    point's cells, at the reference's measured cell-iterations/s per host
    core, scheduled longest first over the cores it was measured on."""
    cores = int(cpu["cores"])
    rate = float(cpu["value"]) / cores  # cell-iterations/s of one core
    loads = [0.0] * cores
    for work in sorted((p["iterations"] * p["cells"] / rate for p in points), reverse=True):
        k = loads.index(min(loads))
        loads[k] += work
    wall = max(loads)
    return {"solves_per_min": 60.0 * len(points) / wall, "wall_s": wall, "cores": cores,
            "basis": "estimate: plain-form iterations x cells per point at the reference's measured "
                     "cell-iterations/s per core (cpu_baseline), longest first over the cores; not a timed run"}


def polar_to_tolerance(cb, tolerance, cap, chunk, forms=("plain", "mixed"), csv_prefix=""):
    """The 24 solves of the batched polar, each solved to worst residual <
    `tolerance` (or `cap` iterations) in the solve engine, in each form:
    solves/min, time-to-convergence percentiles, and per solve the mixed
    form's Cl/Cd/Cm and L-inf Cp differences from the plain FP64 form (which
    the parity tests tie to the FP64 oracle)."""
    out = {"workload": POLAR_NAME, "tolerance": tolerance, "cap": cap, "chunk": chunk}
    runs = {}
    for form in forms:
        reqs = _polar_requests(cb, tolerance, cap, 0 if form == "plain" else 1)
        engine = cb.Engine(chunk=chunk)
        t0 = time.perf_counter()
        results = sorted(engine.run(reqs), key=lambda r: r.id)
        wall = time.perf_counter() - t0
        cps = {r.id: engine.surface(r.id) for r in results if r.status != 2}
        engine.close()
        runs[form] = (results, cps)
        summary = _summarise(results, wall, cb)
        if csv_prefix:
            sweep = [r for r in results if reqs[r.id].designation.decode() == "2412"]
            with open(f"{csv_prefix}_{form}.csv", "w") as fh:
                fh.write(cb.polar_csv(sweep, [reqs[r.id].alpha_deg for r in sweep], "NACA 2412",
                                      "768x192", 3e6, 1.0))
        summary["points"] = [{"alpha": reqs[r.id].alpha_deg, "section": reqs[r.id].designation.decode(),
                              "cells": r.cells, "status": cb.STATUS_NAMES[r.status],
                              "iterations": r.iterations, "ctas": r.cluster_size,
                              "cl": r.lift_coefficient, "cd": r.drag_coefficient,
                              "cm": r.moment_coefficient} for r in results]
        out[form] = summary
    if len(forms) == 2:
        (rp, cpp), (rm, cpm) = runs["plain"], runs["mixed"]
        rows = []
        for a, b in zip(rp, rm):
            row = {"id": a.id, "dcl": abs(b.lift_coefficient - a.lift_coefficient),
                   "dcd": abs(b.drag_coefficient - a.drag_coefficient),
                   "dcm": abs(b.moment_coefficient - a.moment_coefficient),
                   "status_plain": cb.STATUS_NAMES[a.status], "status_mixed": cb.STATUS_NAMES[b.status],
                   "iterations_plain": a.iterations, "iterations_mixed": b.iterations}
            if a.id in cpp and b.id in cpm and len(cpp[a.id]) == len(cpm[b.id]):
                row["dcp_inf"] = float(np.max(np.abs(cpm[b.id] - cpp[a.id])))
            rows.append(row)
        both = [r for r, a, b in zip(rows, rp, rm) if a.status == 0 and b.status == 0]
        out["mixed_vs_plain"] = {
            "solves_per_min_ratio": out["mixed"]["solves_per_min"] / out["plain"]["solves_per_min"],
            "max_dcl": max(r["dcl"] for r in rows), "max_dcd": max(r["dcd"] for r in rows),
            "max_dcm": max(r["dcm"] for r in rows),
            "max_dcp_inf": max((r.get("dcp_inf", 0.0) for r in rows), default=None),
            "both_converged": len(both),
            "max_dcl_both_converged": max((r["dcl"] for r in both), default=None),
            "max_dcd_both_converged": max((r["dcd"] for r in both), default=None),
            "per_solve": rows}
    return out


def run_polar(args) -> None:
    """The batched polar solved to convergence, alone (its JSON line only)."""
    import torch
    torch.cuda.set_device(0)
    import cfd_b200 as cb
    cb.set_device(0)
    forms = ("plain", "mixed") if args.precision == "both" else (args.precision,)
    print(json.dumps(polar_to_tolerance(cb, args.tolerance, args.cap, args.chunk, forms, args.csv)),
          flush=True)


def run_settled(args) -> None:
    """Accuracy of the mixed form where it can be judged: at the two forms'
    settled fixed points. NACA 0012 SST Re 1e6 alpha 0 and 4 on 384x96 and
    NACA 2412 SST Re 3e6 alpha 2 and 6 on 768x192 run in the mixed form from
    the uniform start until Cl moves by less than 1e-7 and Cd by less than
    1e-8 over 1,000 iterations (or --cap iterations); the plain FP64 form then
    continues from the mixed form's state to its own settled point by the
    same rule, and the forces and Cp of the two are compared. (At the
    production tolerance 1e-6 neither form's Cl has settled: it still moves
    by ~1e-2 there, so differences at that tolerance measure convergence, not
    precision.)"""
    import torch
    torch.cuda.set_device(0)
    import cfd_b200 as cb
    cb.set_device(0)
    cap = args.cap if args.cap > 4000 else 60000
    window, cl_move, cd_move = 1000, 1e-7, 1e-8
    cases = [("0012", 0.0, 1e6, "medium", 1e-5), ("0012", 4.0, 1e6, "medium", 1e-5),
             ("2412", 2.0, 3e6, "fine", 5e-6), ("2412", 6.0, 3e6, "fine", 5e-6)]
    fields = ("U", "V", "P", "MASS_FLUX", "K", "OMEGA", "MUT", "MU_EFF")
    meshes = {}

    def make(k, precision):
        des, alpha, re, level, fl = cases[k]
        mesh = _mesh(cb, des, level, fl, meshes)
        s = cb.SimpleSolver.create(mesh, cb.freestream_conditions(mesh, 1.0, alpha),
                                   cb.Settings.defaults(inflow_intensity=INTENSITY,
                                                        inflow_viscosity_ratio=VISCOSITY_RATIO,
                                                        precision=precision))
        s.set_turbulence_model(cb.MODEL_SST)
        return s

    def settle(solvers):
        """Iterate a batch in windows until every solve's Cl and Cd have
        settled (or the cap); returns iterations and whether each settled."""
        batch = cb.Batch(solvers)
        last = [None] * len(solvers)
        done = [False] * len(solvers)
        taken = 0
        while taken < cap and not all(done):
            batch.iterate(window)
            taken += window
            for k, s in enumerate(solvers):
                f, _, _ = s.forces(1.0, cases[k][1], 1.0)
                now = (f.lift_coefficient, f.drag_coefficient)
                if last[k] is not None:
                    done[k] = abs(now[0] - last[k][0]) < cl_move and abs(now[1] - last[k][1]) < cd_move
                last[k] = now
        batch.close()
        return taken, done

    out = {"workload": "settled: NACA0012 SST Re1e6 384x96 alpha 0/4, NACA2412 SST Re3e6 768x192 alpha 2/6",
           "rule": f"Cl moves < {cl_move:g} and Cd < {cd_move:g} over {window} iterations", "cap": cap}
    with _cluster_env(MIXED_CLUSTER):
        mixed = [make(k, 1) for k in range(len(cases))]
    for k, s in enumerate(mixed):
        des, alpha, re, level, fl = cases[k]
        s.initialise(*cb.uniform_field(s.mesh, 1.0, alpha, 1.0, re))
    t0 = time.perf_counter()
    it_m, ok_m = settle(mixed)
    wall_m = time.perf_counter() - t0
    plain = [make(k, 0) for k in range(len(cases))]
    for k, (m, p) in enumerate(zip(mixed, plain)):
        p.initialise(*cb.uniform_field(p.mesh, 1.0, cases[k][1], 1.0, cases[k][2]))
        p.load_state(**{f.lower(): m.read(f) for f in fields})
    t0 = time.perf_counter()
    it_p, ok_p = settle(plain)
    wall_p = time.perf_counter() - t0
    rows = []
    for k, (m, p) in enumerate(zip(mixed, plain)):
        fm, cpm, _ = m.forces(1.0, cases[k][1], 1.0)
        fp, cpp, _ = p.forces(1.0, cases[k][1], 1.0)
        rows.append({"case": f"{cases[k][0]} alpha {cases[k][1]:g} {cases[k][3]}",
                     "settled_mixed": ok_m[k], "settled_plain": ok_p[k],
                     "cl_plain": fp.lift_coefficient, "cd_plain": fp.drag_coefficient,
                     "dcl": abs(fm.lift_coefficient - fp.lift_coefficient),
                     "dcd": abs(fm.drag_coefficient - fp.drag_coefficient),
                     "dcm": abs(fm.moment_coefficient - fp.moment_coefficient),
                     "dcp_inf": float(np.max(np.abs(cpm - cpp)))})
    out["mixed"] = {"iterations": it_m, "wall_s": wall_m}
    out["plain_from_mixed"] = {"iterations": it_p, "wall_s": wall_p}
    out["mixed_vs_plain"] = rows
    for s in mixed + plain:
        s.close()
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


def serve(cb, rate, requests, seed, precision, tolerance, cap, chunk) -> dict:
    """One serving run: the seeded Poisson stream submitted to the engine in
    real time (engine clock), stepped until every request has finished.
    Time to convergence is finished - submitted per request, so it includes
    queueing; the served rate says whether the GPU kept up with the offered
    one (when it does not, the queue grows and the percentiles measure it)."""
    stream = serving_stream(requests, rate, seed)
    settings = cb.Settings.defaults(inflow_intensity=INTENSITY, inflow_viscosity_ratio=VISCOSITY_RATIO,
                                    precision=1 if precision == "mixed" else 0)
    engine = cb.Engine(chunk=chunk, tuned=True)  # a saturated GPU: the occupancy tuner
    t0 = engine.clock()
    submitted, results = 0, []
    wall0 = time.perf_counter()
    while len(results) < len(stream):
        now = engine.clock() - t0
        while submitted < len(stream) and stream[submitted][0] <= now:
            _, des, alpha, re, level, fl = stream[submitted]
            sp, wp, npn = GRIDS[level]
            engine.submit(cb.request(des, alpha, re, tolerance=tolerance, max_iterations=cap,
                                     surface_points=sp, wake_points=wp, normal_points=npn,
                                     first_layer_height=fl, settings=settings))
            submitted += 1
        active, queued = engine.step()
        results.extend(engine.results())
        if active == 0 and queued == 0 and submitted < len(stream):
            time.sleep(max(0.0, min(0.05, stream[submitted][0] - (engine.clock() - t0))))
    wall = time.perf_counter() - wall0
    engine.close()
    out = _summarise(results, wall, cb)
    served = len(results) / wall
    out.update({"workload": f"serve: Poisson lambda={rate:g}/s, {requests} NACA 4-digit SST "
                            f"requests (seed {seed}), meshes 192x48/384x96/768x192 at "
                            "0.5/0.35/0.15", "precision": precision,
                "offered_per_s": rate, "served_per_s": served, "saturated": served < 0.9 * rate,
                "tolerance": tolerance, "cap": cap, "chunk": chunk})
    return out


def run_serve(args) -> None:
    """configs[4] at its own rate (lambda = 4/s), then, when the GPU could not
    keep up with it, the same kind of stream at 70 % of the rate it served,
    where the latency percentiles measure the solves rather than the queue."""
    import torch
    torch.cuda.set_device(0)
    import cfd_b200 as cb
    cb.set_device(0)
    precision = "mixed" if args.precision == "mixed" else "plain"
    out = serve(cb, args.rate, args.requests, args.seed, precision, args.tolerance, args.cap, args.chunk)
    if out["saturated"]:
        rate = 0.7 * out["served_per_s"]
        out["sustainable"] = serve(cb, rate, max(64, args.requests // 4), args.seed + 1, precision,
                                   args.tolerance, args.cap, args.chunk)
    print(json.dumps(out), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-convergence", action="store_true",
                    help="skip solving the polar to convergence in both forms")
    ap.add_argument("--no-mixed", action="store_true",
                    help="skip timing the mixed form's batch")
    ap.add_argument("--workload", choices=("batch", "c2", "polar", "serve", "settled"), default="batch",
                    help="batch: the benchmark line, the 24-solve polar in one launch per step "
                         "(default); c2: the 384x96 pair; polar / serve / settled: engine workloads")
    ap.add_argument("--solves", type=int, default=None,
                    help="batch: time only the first N solves of the polar (a smaller case "
                         "for profiling captures; the benchmark line uses all 24)")
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
                    help="batch / c2: replay each step's launch from a CUDA graph")
    ap.add_argument("--form", choices=("plain", "mixed"), default="plain",
                    help="batch / c2: the form the benchmark line times (plain FP64 by default)")
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
