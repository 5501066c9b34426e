#!/usr/bin/env python
"""Throughput of the B200 electrostatic PIC step (particle-steps/s incl. the
Poisson multigrid solve), on the 2-D bounded two-species plasma:

  1024 x 1024 cells, dx = 1 (Debye length), grounded Dirichlet walls and
  absorbing particle boundaries; 256 particles/cell/species (536,870,912
  particles); electrons vth = 1, ions m = 1836 at equal temperature; uniform
  positions, Maxwellian velocities; leapfrog push, dt = 0.1/omega_p; FP32
  push with int32 cell + FP32 offset; FP32 V(2,2) multigrid inside FP64
  refinement to 1e-8 relative residual.

One step = rho from the exact charge accumulators -> multigrid solve -> fused
gather/push/boundary/deposit -> stable re-sort by cell (every
--sort-interval steps).  Inputs are larger than L2, so no flush is needed.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs independent replicas (one per GPU, different seeds): the path has
no data-path exchange between GPUs.  `--impl reference` times the CPU
restatement of PSuM's algorithm (oracle/, FP64, OpenMP on all host cores) on
a bounded sample of the same workload.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CELLS = 1024
PPC = 256
DT = 0.1
MASS_RATIO = 1836.0
SEED = 20261203 + 2
MG_OPTIONS = (f"I {CELLS + 1} J {CELLS + 1} K 1 depth 5 pre_relax 2 post_relax 2 max_cycles 16 "
              f"correction_interval 2 tol 1e-8")
BYTES_PER_PARTICLE = 24          # int32 cell + 2 FP32 offsets + 3 FP32 velocities (2D3V mixed)
COMPARE_STEPS = 3                # steps from the common initial state before the mixed/FP64 field comparison
FP64_SORT_INTERVAL = 4           # the FP64 comparison run: in-place push, stable re-sort every 4 steps
FP64_BYTES_PER_PARTICLE = 44     # FP64 2 positions + 3 velocities + int32 cell key (2D3V FP64)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ppc", type=int, default=PPC, help="particles per cell per species")
    ap.add_argument("--cells", type=int, default=CELLS)
    ap.add_argument("--sort-interval", type=int, default=1)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 GPU run and the field comparison")
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c4", "c5", "bspline"],
                    help="c2 (default): the bench line; c1/c3/c5: the other plasmas of the scope table; "
                         "c4: the differentiable run (forward and adjoint); bspline: B-spline gather + deposit")
    ap.add_argument("--order", type=int, default=2, help="B-spline order of the bspline workload (1-4)")
    ap.add_argument("--bs-cells", type=int, default=1023, help="cells per axis of the bspline workload")
    ap.add_argument("--wl-cells", type=int, default=0, help="cells per axis of c1/c3/c5 (default: the workload's)")
    ap.add_argument("--wl-ppc", type=int, default=0, help="particles per cell of c1/c3 (default: the workload's)")
    ap.add_argument("--mg-extra", default="", help="extra multigrid options (e.g. 'graph 0' to launch the solve's "
                    "kernels one by one, which profilers need)")
    return ap.parse_args()


# ----------------------------------------------------------------- helpers --
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.file = None

    def __enter__(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "200"], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.file is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.file.flush()
        rows = []
        with open(self.file.name) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------- replicas --
def replica_seed(rank):
    """Seed of one replica: replicas are independent runs of the workload."""
    return SEED + 1000 * rank


def max_over_ranks(value, dist, device):
    """The largest of the ranks' values (all ranks take this collective)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(particles_per_rank, world, steps, ms_max):
    """Whole-job particle-steps/s: all ranks' particle-steps over the slowest
    rank's time."""
    return particles_per_rank * world * steps / (ms_max * 1e-3)


def make_species_device(torch, gen, n, cells, vth, device):
    pos = torch.rand((2, n), generator=gen, device=device, dtype=torch.float64) * cells
    vel = torch.randn((3, n), generator=gen, device=device, dtype=torch.float64) * vth
    return pos, vel


def mg_options(cells, extra=""):
    opts = MG_OPTIONS.replace(f"I {CELLS + 1} J {CELLS + 1}", f"I {cells + 1} J {cells + 1}")
    return f"{opts} {extra}".strip()


def build_problem(torch, P, cells, ppc, seed, device, sort_interval, mg_extra="", precision=None,
                  backend="cuda_multigrid32f_gpu"):
    """Context + solver for the bounded two-species plasma (particles are
    loaded by the caller)."""
    n = cells * cells * ppc
    w = 1.0 / ppc
    ctx = P.ParticleContext((cells, cells), (0.0, 0.0), (float(cells), float(cells)), (0, 0),
                            P.MIXED if precision is None else precision)
    # every step also computes the energy and charge diagnostics (TSI/main.cpp:132-146) inside its kernels
    ctx.set_options(f"sort_interval {sort_interval} diagnostics 1")
    e = ctx.add_species(-1.0, 1.0, w, n)
    i = ctx.add_species(1.0, MASS_RATIO, w, n)
    grid = P.simple_grid((0.0, 0.0), (float(cells), float(cells)), (cells, cells))
    ps = P.Poisson_solver_2d()
    opts = mg_options(cells, mg_extra)
    ps.set_options(opts)
    ps.init(backend, grid, P.Poisson_solver_2d.Cartesian,
            [P.Dirichlet_line(grid, d, 0.0) for d in "NSEW"], 1.0)
    ps.make_righthand_item()
    return ctx, (e, i), ps, n, w


def roofline_block(push_ms_per_step, n_total, peak, peak_kind, traffic):
    """Roofline of the dominant work: the fused sorted step of both species
    (gather + push + boundary + deposit + stable re-sort), whose algorithmic
    bytes are one read and one write of every particle's state (2 x 24 B)."""
    algo = n_total * 2 * BYTES_PER_PARTICLE
    achieved = algo / (push_ms_per_step * 1e-3) / 1e9
    return {"bound": "hbm",
            "kernel": "fused sorted step: k_cls_pass1 + k_cls_offsets + scan + k_cls_pass2, both species",
            "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
            "peak_kind": peak_kind, "algorithmic_bytes_per_step": algo,
            "traffic": None if traffic is None else int(traffic * n_total)}


def step_algorithmic_bytes(n_total, cells, cycles, refinements, pre=2, post=2):
    """B_step = N_p * 2 S_p + B_grid with B_grid = N_nodes (b_phi + b_rho)
    + n_VC c_d N_nodes (pre + post + 3) 3 b_f + n_ref N_nodes (2*8 + 4):
    compulsory traffic of the particle state, the FP64 fields, the FP32
    V-cycles (c_d = 4/3, the 2-D level sum) and the FP64 refinements."""
    nodes = (cells + 1) ** 2
    grid = nodes * 16 + cycles * (4.0 / 3.0) * nodes * (pre + post + 3) * 3 * 4 + refinements * nodes * 20
    return n_total * 2 * BYTES_PER_PARTICLE + int(grid)


def measured_traffic_per_particle():
    """DRAM bytes (read + write) per particle of the fused sorted step from
    the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", "fused_step_traffic.txt")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        for line in f:
            if line.startswith("bytes_per_particle:"):
                return float(line.split(":", 1)[1])
    return None


def step_roofline(n_total, cells, stats, ms_per_step, peak):
    b = step_algorithmic_bytes(n_total, cells, stats["cycles"], stats["refinements"])
    achieved = b / (ms_per_step * 1e-3) / 1e9
    return {"algorithmic_bytes": b, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4)}


def workload_config(args, world=1):
    return {"workload": "2D bounded two-species plasma, mixed precision",
            "grid_cells": [args.cells, args.cells], "particles": 2 * args.cells * args.cells * args.ppc,
            "ppc_per_species": args.ppc, "mass_ratio": MASS_RATIO, "dt": DT, "mg": mg_options(args.cells, args.mg_extra),
            "sort_interval": args.sort_interval, "parallelism": "replicas" if world > 1 else "single GPU",
            "l2_policy": "inputs larger than L2 (state 12.9 GB)"}


# ------------------------------------------------------------ CPU baseline --
CPU_CELLS = 128   # sub-domain of the CPU baseline (whole steps, same plasma)


class CpuRun:
    """Whole steps of the bounded two-species plasma on the host: the FP64 CPU
    restatement of PSuM's algorithm (oracle/, OpenMP on all host cores) on a
    CPU_CELLS x CPU_CELLS-cell sub-domain of the same plasma (same particles per
    cell, dx, dt, walls, mass ratio): deposit -> FP32-in-FP64 multigrid solve
    with the GPU run's options and stopping rule (V(2,2), correction interval
    2, relative residual 1e-8, at most 16 cycles, previous phi as the initial
    guess) -> push with absorbing walls.  Each step is timed whole; nothing is
    extrapolated."""

    def __init__(self, cells, ppc, seed):
        import numpy as np
        from oracle import oracle as O
        from psum_b200.field_solver import Dirichlet_line, simple_grid
        self.O, self.np = O, np
        rng = np.random.default_rng(seed)
        self.cells = cells
        self.g = O.make_grid((cells, cells), (0.0, 0.0), (float(cells), float(cells)), (0, 0))
        grid = simple_grid((0.0, 0.0), (float(cells), float(cells)), (cells, cells))
        self.fixed = np.unique(np.concatenate([Dirichlet_line(grid, d, 0.0)[0] for d in "NSEW"])).astype(np.int64)
        r, c, v = O.poisson_assemble((cells, cells), (0, 0), (cells, cells), 1.0, self.fixed)
        self.nn = (cells + 1) ** 2
        depth = max(2, min(5, int(math.log2(cells)) - 2))
        self.mg = O.Multigrid(r, c, v, self.nn, cells + 1, cells + 1, 1, depth)
        self.w = 1.0 / ppc
        n = cells * cells * ppc
        self.n_total = 2 * n
        self.species = []
        for q, m, vth in ((-1.0, 1.0, 1.0), (1.0, MASS_RATIO, 1.0 / math.sqrt(MASS_RATIO))):
            pos = rng.uniform(0.0, cells, size=(2, n))
            vel = rng.normal(0.0, vth, size=(3, n))
            self.species.append([q, m, pos, vel])
        self.phi = np.zeros(self.nn)
        self.last = None

    def step(self):
        O, np = self.O, self.np
        rho = np.zeros(self.nn)
        for q, m, pos, vel in self.species:
            rho += O.deposit(self.g, pos, q * self.w, self.nn)
        b = rho.copy()
        b[self.fixed] = 0.0
        self.phi, hist = self.mg.solve_mixed_tol(b, self.phi, 16, 2, 2, 2, 1e-8)
        for sp in self.species:
            sp[2], sp[3], _ = O.push(self.g, sp[2], sp[3], self.phi, sp[0] / sp[1], DT)
        self.last = {"batches": int(len(hist)), "rel_residual": float(hist[-1]) if len(hist) else None}

    def describe(self, steps):
        return (f"{steps} whole steps (deposit + FP32-in-FP64 multigrid solve to 1e-8 + push) of the same plasma "
                f"on a {self.cells}x{self.cells}-cell sub-domain, {self.n_total} particles (2 species, same particles "
                f"per cell); last solve {self.last['batches']} refinements, relative residual "
                f"{self.last['rel_residual']:.1e}")


def cpu_baseline(ppc, warmup=1, steps=3):
    """Throughput of whole CPU steps (CpuRun) in particle-steps/s."""
    run = CpuRun(CPU_CELLS, ppc, SEED)
    for _ in range(warmup):
        run.step()
    t0 = time.perf_counter()
    for _ in range(steps):
        run.step()
    dt = time.perf_counter() - t0
    return {"value": run.n_total * steps / dt, "unit": "particle-steps/s", "cores": os.cpu_count(), "kind": "port",
            "sample": run.describe(steps), "ms_per_step": 1e3 * dt / steps}


# --------------------------------------------------------------- main arm --
def run_ours(args, rank, world, dist):
    import numpy as np
    import torch

    import psum_b200 as P
    torch.cuda.set_device(rank % torch.cuda.device_count())
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.Stream()
    cells, ppc = args.cells, args.ppc
    gen = torch.Generator(device=dev)
    gen.manual_seed(replica_seed(rank))

    ctx, (e, i), ps, n, w = build_problem(torch, P, cells, ppc, SEED + rank, dev, args.sort_interval, args.mg_extra)
    ctx.set_stream(stream)
    nn = (cells + 1) ** 2
    rho = torch.zeros(nn, dtype=torch.float64, device=dev)
    phi = torch.zeros(nn, dtype=torch.float64, device=dev)
    vth_i = 1.0 / np.sqrt(MASS_RATIO)
    init = []   # the FP64 initial state, kept for the FP64 run
    for sp, vth in ((e, 1.0), (i, vth_i)):
        pos, vel = make_species_device(torch, gen, n, cells, vth, dev)
        ctx.load(sp, pos, vel)
        init.append((pos, vel))
    torch.cuda.synchronize()
    ctx.sort()
    ctx.deposit()

    def step():
        ctx.step(ps.backend, 0.0, rho, phi, DT)

    # the first COMPARE_STEPS steps (untimed) give the fields compared with
    # the FP64 run from the same initial state
    for _ in range(COMPARE_STEPS):
        step()
    torch.cuda.synchronize()
    rho_mixed, phi_mixed = rho.clone(), phi.clone()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    ctx.get_timing(reset=True)
    ctx.set_timing(True)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = P.lib().psum_kernel_launches()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clk:
        with torch.cuda.stream(stream):
            start.record(stream)
            for _ in range(args.steps):
                step()
            ctx.join()   # the last step's deferred second pass is inside the timed region
            stop.record(stream)
        torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    launches = P.lib().psum_kernel_launches() - launches0
    ms = start.elapsed_time(stop)
    phases = ctx.get_timing(reset=True)
    ctx.set_timing(False)
    stats = ps.backend.last_stats()
    step_diag = ctx.step_diagnostics(1.0)   # the last timed step's own diagnostics
    n_valid = sum(ctx.count(sp)[1] for sp in (e, i))
    diag = ctx.diagnostics(phi, 1.0)
    clocks = clk.summary()

    ms_max = max_over_ranks(ms, dist, dev)

    fp64 = None
    if not args.no_fp64:
        del ctx, ps
        torch.cuda.empty_cache()
        fp64 = run_fp64(args, torch, P, dev, init, rho_mixed, phi_mixed)
    del init
    torch.cuda.empty_cache()

    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, torch, P, dev, rank, dist)

    if rank != 0:
        return None
    n_total = 2 * n
    value = replica_value(n_total, world, args.steps, ms_max)
    peak, peak_kind = measured_peaks()
    push_ms = phases["push"][0] / max(phases["push"][1], 1)
    traffic = measured_traffic_per_particle()
    line = {
        "metric": "particle-steps/s incl. Poisson MG, mixed-prec vs FP64 on GPU at stated error",
        "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 push / f32-in-f64 MG", "data": "synthetic",
        "config": workload_config(args, world),
        "roofline": roofline_block(push_ms, n_total, peak, peak_kind, traffic),
        "phase_ms_per_step": {k: round(v[0] / max(v[1], 1), 4) for k, v in phases.items()},
        "step_roofline": step_roofline(n_total, cells, stats, ms_max / args.steps, peak),
        "mg_last_solve": stats, "valid_particles_end": n_valid, "charge_end": diag["charge"],
        "step_diagnostics": {"kinetic_electrons": step_diag["kinetic"][0], "kinetic_ions": step_diag["kinetic"][1],
                             "field_energy": step_diag["field"], "charge_of_density": step_diag["charge"],
                             "definition": "computed inside every timed step (push, edge and density kernels), "
                                           "FP64 fixed-order sums; values of the last step"},
        "gpu_launches": int(launches), "clocks": clocks,
    }
    if fp64 is not None:
        fp64["mixed_over_fp64"] = round(value / fp64["value"], 3)   # the >= 2x target of the mixed method
        line["fp64_gpu"] = fp64
    if e2e is not None:
        line["e2e"] = e2e
    if not args.no_cpu_baseline:
        cb = cpu_baseline(ppc)
        cb.pop("ms_per_step", None)
        line["cpu_baseline"] = cb
    return line


def run_fp64(args, torch, P, dev, init, rho_mixed, phi_mixed):
    """The same workload in FP64 on the GPU (FP64 particle state, FP64
    multigrid V-cycles): throughput over K timed steps, and the relative field
    error of the mixed run against it after COMPARE_STEPS steps from the same
    initial state."""
    cells, ppc = args.cells, args.ppc
    ctx, (e, i), ps, n, w = build_problem(torch, P, cells, ppc, SEED, dev, FP64_SORT_INTERVAL, args.mg_extra,
                                          precision=P.FP64, backend="cuda_multigrid64_gpu")
    ctx.set_options("fp64_fma 1")   # the contracted FP64 kernels (the bit-exact build is the parity checker)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream)
    nn = (cells + 1) ** 2
    rho = torch.zeros(nn, dtype=torch.float64, device=dev)
    phi = torch.zeros(nn, dtype=torch.float64, device=dev)
    for sp, (pos, vel) in zip((e, i), init):
        ctx.load(sp, pos, vel)
    torch.cuda.synchronize()
    ctx.sort()
    ctx.deposit()
    for _ in range(COMPARE_STEPS):
        ctx.step(ps.backend, 0.0, rho, phi, DT)
    torch.cuda.synchronize()

    def rel(a, b):
        return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))

    err = {"after_steps": COMPARE_STEPS, "phi_rel_l2": rel(phi_mixed, phi), "rho_rel_l2": rel(rho_mixed, rho),
           "phi_rel_max": float((phi_mixed - phi).abs().max() / phi.abs().max())}
    for _ in range(args.warmup):
        ctx.step(ps.backend, 0.0, rho, phi, DT)
    torch.cuda.synchronize()
    ctx.get_timing(reset=True)
    ctx.set_timing(True)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        start.record(stream)
        for _ in range(args.steps):
            ctx.step(ps.backend, 0.0, rho, phi, DT)
        ctx.join()
        stop.record(stream)
    torch.cuda.synchronize()
    ms = start.elapsed_time(stop) / args.steps
    phases = ctx.get_timing(reset=True)
    del ctx, ps
    torch.cuda.empty_cache()
    peak, peak_kind = measured_peaks()
    algo = 2 * n * 2 * FP64_BYTES_PER_PARTICLE
    return {"value": 2 * n * args.steps / (ms * args.steps * 1e-3), "unit": "particle-steps/s", "ms_per_step": ms,
            "definition": f"FP64 particle state and FP64 V-cycles (cuda_multigrid64_gpu, same options), "
                          f"contracted FP64 kernels, in-place push with deposit, stable sort every "
                          f"{FP64_SORT_INTERVAL} steps, diagnostics in every step",
            "phase_ms_per_step": {k: round(v[0] / max(v[1], 1), 4) for k, v in phases.items()},
            "roofline": {"bound": "hbm", "algorithmic_bytes_per_step": algo,
                         "definition": "one read and one write of every particle's FP64 state and key (2 x 44 B)",
                         "achieved": round(algo / (ms * 1e-3) / 1e9, 1), "peak": peak, "peak_kind": peak_kind,
                         "frac": round(algo / (ms * 1e-3) / 1e9 / peak, 4)},
            "field_error_of_mixed": err}


def run_e2e(args, torch, P, dev, rank, dist):
    """The same job end to end through the C ABI from pinned host buffers:
    H2D of the initial particle state (FP64 SoA, as PSuM's particles are
    FP64), then K steps, each followed by a D2H read of the loss counters,
    then a D2H read of phi."""
    import numpy as np
    cells, ppc = args.cells, args.ppc
    n = cells * cells * ppc
    need = 2 * n * 5 * 8
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except Exception:
        avail = 0
    if avail and avail < 1.5 * need:
        return {"value": None, "unit": "particle-steps/s",
                "skipped": f"host RAM {avail / 1e9:.0f} GB < 1.5 x {need / 1e9:.0f} GB pinned input"}
    gen = torch.Generator(device=dev)
    gen.manual_seed(SEED + 7 + 1000 * rank)
    host = []
    for vth in (1.0, 1.0 / np.sqrt(MASS_RATIO)):
        pos, vel = make_species_device(torch, gen, n, cells, vth, dev)
        hp = torch.empty(pos.shape, dtype=torch.float64, pin_memory=True)
        hv = torch.empty(vel.shape, dtype=torch.float64, pin_memory=True)
        hp.copy_(pos)
        hv.copy_(vel)
        del pos, vel
        host.append((hp, hv))
    torch.cuda.synchronize()
    ctx, (e, i), ps, n, w = build_problem(torch, P, cells, ppc, SEED + rank, dev, args.sort_interval, args.mg_extra)
    nn = (cells + 1) ** 2
    rho = torch.zeros(nn, dtype=torch.float64, device=dev)
    phi = torch.zeros(nn, dtype=torch.float64, device=dev)
    phi_host = torch.empty(nn, dtype=torch.float64, pin_memory=True)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for sp, (hp, hv) in zip((e, i), host):
        P.check(P.lib().psum_pic_load(ctx.handle, sp, n, hp.data_ptr(), hv.data_ptr()))
    ctx.sort()
    ctx.deposit()
    losses_total = 0
    for _ in range(args.steps):
        ctx.step(ps.backend, 0.0, rho, phi, DT)
        losses_total += int(ctx.losses(reset=True).sum())
    phi_host.copy_(phi)
    torch.cuda.synchronize()
    sec = max_over_ranks(time.perf_counter() - t0, dist, dev)
    world = dist.get_world_size() if dist is not None else 1
    h2d = 2 * n * 5 * 8
    d2h = args.steps * 2 * 2 * 2 * 8 + nn * 8
    del ctx, ps, host
    return {"value": replica_value(2 * n, world, args.steps, sec * 1e3), "unit": "particle-steps/s",
            "h2d_bytes_per_step": h2d // args.steps, "d2h_bytes_per_step": d2h // args.steps,
            "wall_s": sec, "definition": "whole job: H2D of the FP64 particle state, then K steps with a D2H "
                                         "of the loss counters after each, then D2H of phi"}


# --------------------------------------------------- other workloads ---
WORKLOADS = {
    # name: (dim, cells, ppc or total, precision, depth, tol, dt, steps in the config)
    "c1": dict(dim=2, cells=63, ppc=64, precision="fp64", depth=4, tol=1e-10, dt=0.1,
               desc="2D periodic electrostatic plasma, FP64 plain method: 64x64 wrapping nodes, 64 e-/cell, "
                    "1% mode-1 density perturbation, uniform ion background"),
    "c3": dict(dim=3, cells=255, ppc=32, precision="mixed", depth=5, tol=1e-8, dt=0.05, gauge="mean",
               desc="3D periodic two-stream, mixed precision: 256^3 wrapping nodes, 32 e-/cell in two beams at "
                    "+/-5 vth along x (dt 0.05: the beams move a quarter cell per step)"),
    "c5": dict(dim=3, cells=511, total=1_000_000_000, precision="mixed", depth=6, tol=1e-8, dt=0.1, gauge="mean",
               desc="3D clustered-load stress: 512^3 wrapping nodes, 1e9 e- from a Gaussian blob "
                    "(sigma = 0.05 L) drifting at 2 vth along z"),
    "c4": dict(dim=2, cells=255, ppc=64, precision="mixed", depth=5, tol=1e-10, dt=0.1,
               desc="2D differentiable run: 256^2 wrapping nodes, 64 e-/cell, Landau damping (5% mode-1), "
                    "100 steps, loss = field energy at the final step, gradients by the adjoint with "
                    "checkpoints every 10 steps"),
}


def periodic_problem(P, w, mg_extra=""):
    """Grid (TSI idiom: lower corner at dx/2), gauge, solver.  The gauge is
    the TSI pinned node, or for the 3D workloads the mean-zero potential
    (solver option null_space 1): in FP32 V-cycles the pinned operator's
    lowest mode, eigenvalue ~ 1/nodes, falls below single-precision
    resolution at 256^3 and the refinement stalls near 1e-4."""
    dim, cells = w["dim"], w["cells"]
    nodes = cells + 1
    lo, hi = (0.5,) * dim, (cells + 0.5,) * dim
    grid = P.simple_grid(lo, hi, (cells,) * dim)
    opts = (f"I {nodes} J {nodes} K {nodes if dim == 3 else 1} depth {w['depth']} pre_relax 2 post_relax 2 "
            f"max_cycles 24 correction_interval 2 tol {w['tol']} periodic_I 1 periodic_J 1"
            + (" periodic_K 1" if dim == 3 else "") + (" null_space 1" if w.get("gauge") == "mean" else "")
            + (f" {mg_extra}" if mg_extra else ""))
    fixed = [] if w.get("gauge") == "mean" else [P.Dirichlet_nodes(grid, [(0,) * dim], 0.0)]
    backend = "cuda_multigrid64_gpu" if w["precision"] == "fp64" else "cuda_multigrid32f_gpu"
    return grid, opts, fixed, backend


def periodic_initial_state(torch, w, gen, dev):
    """Positions (dim, n) and velocities (3, n), FP64 on the device."""
    dim, L = w["dim"], w["cells"] + 1.0
    name = w["name"]
    n = w["total"] if "total" in w else int(L ** dim * w["ppc"])
    if name == "c5":
        pos = torch.randn((dim, n), generator=gen, device=dev, dtype=torch.float64) * (0.05 * L) + L / 2
        pos = torch.remainder(pos, L)
        vel = torch.randn((3, n), generator=gen, device=dev, dtype=torch.float64)
        vel[2] += 2.0
    else:
        pos = torch.rand((dim, n), generator=gen, device=dev, dtype=torch.float64) * L
        if name in ("c1", "c4"):   # mode-1 density perturbation by inverse-CDF displacement in x
            amp = 0.01 if name == "c1" else 0.05
            k = 2 * math.pi / L
            u = pos[0].clone()
            x = u.clone()
            for _ in range(20):
                x -= (x + amp / k * torch.sin(k * x) - u) / (1 + amp * torch.cos(k * x))
            pos[0] = torch.remainder(x, L)
        vel = torch.randn((3, n), generator=gen, device=dev, dtype=torch.float64)
        if name == "c3":           # two counter-streaming beams along x
            vel[0, : n // 2] += 5.0
            vel[0, n // 2:] -= 5.0
    return pos + 0.5, vel, n


def run_workload(args):
    """One of the other plasmas: its own JSON line, same timing rules."""
    import torch

    import psum_b200 as P
    if args.workload == "bspline":
        return run_bspline(args, torch, P)
    w = dict(WORKLOADS[args.workload], name=args.workload)
    if args.wl_cells:   # a smaller (or larger) box of the same plasma, e.g. for profiler captures
        w["cells"] = args.wl_cells
    if args.wl_ppc and "ppc" in w:
        w["ppc"] = args.wl_ppc
    if args.wl_cells or args.wl_ppc:
        w["desc"] += f" [resized: {w['cells'] + 1}^{w['dim']} nodes, {w.get('ppc', '-')} per cell]"
    if args.workload == "c4":
        return run_c4(args, torch, P, w)
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream()
    gen = torch.Generator(device=dev)
    gen.manual_seed(SEED + int(args.workload[1]))
    grid, opts, fixed, backend = periodic_problem(P, w, args.mg_extra)
    pos, vel, n = periodic_initial_state(torch, w, gen, dev)
    L = w["cells"] + 1.0
    precision = P.FP64 if w["precision"] == "fp64" else P.MIXED
    ctx = P.ParticleContext((w["cells"],) * w["dim"], (0.5,) * w["dim"], (w["cells"] + 0.5,) * w["dim"],
                            (1,) * w["dim"], precision)
    sort_interval = args.sort_interval if precision == P.MIXED else 20
    ctx.set_options(f"sort_interval {sort_interval}")
    e = ctx.add_species(-1.0, 1.0, L ** w["dim"] / n, n)
    ctx.load(e, pos, vel)
    del pos, vel
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    ctx.sort()
    ctx.deposit()
    ps = P.Poisson_solver_2d() if w["dim"] == 2 else P.Poisson_solver_3d()
    ps.set_options(opts)
    ps.init(backend, grid, ps.Cartesian, fixed, 1.0)
    ps.make_righthand_item()
    ctx.set_stream(stream)
    nn = grid.n_nodes
    rho = torch.zeros(nn, dtype=torch.float64, device=dev)
    phi = torch.zeros(nn, dtype=torch.float64, device=dev)

    def step():
        ctx.step(ps.backend, 1.0, rho, phi, w["dt"])   # background: the uniform ions

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    ctx.get_timing(reset=True)
    ctx.set_timing(True)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        with torch.cuda.stream(stream):
            start.record(stream)
            for _ in range(args.steps):
                step()
            ctx.join()   # the last step's deferred second pass is inside the timed region
            stop.record(stream)
        torch.cuda.synchronize()
    ms = start.elapsed_time(stop) / args.steps
    phases = ctx.get_timing(reset=True)
    stats = ps.backend.last_stats()
    n_valid = ctx.count(e)[1]
    peak, peak_kind = measured_peaks()
    sp_bytes = (24 if w["dim"] == 2 else 28) if precision == P.MIXED else (44 if w["dim"] == 2 else 52)
    b_step = n * 2 * sp_bytes
    return {"workload": args.workload, "metric": "particle-steps/s incl. Poisson MG",
            "value": n * args.steps / (ms * args.steps * 1e-3), "unit": "particle-steps/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "dtype": "f64" if precision == P.FP64 else "f32 push / f32-in-f64 MG", "data": "synthetic",
            "config": {"workload": w["desc"], "particles": n, "nodes": nn, "dt": w["dt"], "mg": opts,
                       "sort_interval": sort_interval},
            "particle_roofline": {"algorithmic_bytes_per_step": b_step,
                                  "achieved": round(b_step / (ms * 1e-3) / 1e9, 1), "peak": peak,
                                  "frac": round(b_step / (ms * 1e-3) / 1e9 / peak, 4)},
            "phase_ms_per_step": {k: round(v[0] / max(v[1], 1), 4) for k, v in phases.items()},
            "mg_last_solve": stats, "valid_particles_end": n_valid, "clocks": clk.summary()}


BSPLINE_PPC = 64


def run_bspline(args, torch, P):
    """B-spline gather of the potential's gradient and deposit of every
    particle (interp_diff_B_spline + add_back_B_spline at --order) on a
    1024^2-node grid, 64 particles per cell stored cell by cell (the order a
    sorted PIC state has); one step = one gradient gather and one deposit of
    all particles.  Algorithmic bytes: per particle the 16 B position read by
    each kernel and the 16 B gradient written; per node the potential read,
    the fixed-point words zeroed, accumulated and read, and the field
    read-modify-write."""
    from psum_b200 import interp as I
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    cells, ppc, order = args.bs_cells, BSPLINE_PPC, args.order
    nodes = (cells + 1) ** 2
    n = cells * cells * ppc
    gen = torch.Generator(device=dev)
    gen.manual_seed(SEED + 10 + order)
    grid = P.simple_grid((0.5, 0.5), (cells + 0.5, cells + 0.5), (cells, cells))
    cell = torch.arange(n, device=dev, dtype=torch.int64) // ppc
    pos = torch.empty((2, n), dtype=torch.float64, device=dev)
    pos[0] = 0.5 + (cell // cells).double() + torch.rand(n, generator=gen, device=dev, dtype=torch.float64)
    pos[1] = 0.5 + (cell % cells).double() + torch.rand(n, generator=gen, device=dev, dtype=torch.float64)
    del cell
    phi = torch.randn(nodes, generator=gen, device=dev, dtype=torch.float64)
    rho = torch.zeros(nodes, dtype=torch.float64, device=dev)
    scratch = torch.empty(nodes, dtype=torch.int64, device=dev)
    grad = torch.empty((2, n), dtype=torch.float64, device=dev)
    glib = P.lib()
    gd = I.grid_desc(grid)
    import ctypes as C
    stream = torch.cuda.current_stream().cuda_stream

    def gather():
        P.check(glib.psum_interp_diff_bspline(C.byref(gd), order, n, pos.data_ptr(), phi.data_ptr(), grad.data_ptr(),
                                              None, stream))

    def deposit():
        P.check(glib.psum_add_back_bspline(C.byref(gd), order, n, pos.data_ptr(), 1.0 / ppc, rho.data_ptr(),
                                           scratch.data_ptr(), None, stream))

    for _ in range(args.warmup):
        gather()
        deposit()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * args.steps + 1)]
    launches0 = P.lib().psum_kernel_launches()
    with ClockSampler(0) as clk:
        ev[0].record()
        for k in range(args.steps):
            gather()
            ev[2 * k + 1].record()
            deposit()
            ev[2 * k + 2].record()
        torch.cuda.synchronize()
    launches = P.lib().psum_kernel_launches() - launches0
    g_ms = sum(ev[2 * k].elapsed_time(ev[2 * k + 1]) for k in range(args.steps)) / args.steps
    d_ms = sum(ev[2 * k + 1].elapsed_time(ev[2 * k + 2]) for k in range(args.steps)) / args.steps
    ms = g_ms + d_ms
    peak, peak_kind = measured_peaks()
    g_bytes = n * 32 + nodes * 8
    d_bytes = n * 16 + nodes * (8 * 3 + 16)
    line = {"workload": "bspline", "metric": "particle gather+deposit/s", "value": n / (ms * 1e-3),
            "unit": "particles/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"2-D B-spline order {order} gradient gather + deposit, {cells}^2 cells, "
                                   f"{ppc} particles per cell stored cell by cell", "particles": n, "nodes": nodes,
                       "order": order, "l2_policy": f"inputs larger than L2 (positions {n * 16 / 1e9:.2f} GB)"},
            "kernels": {"gather": {"ms": round(g_ms, 4), "algorithmic_bytes": g_bytes,
                                   "achieved_GBs": round(g_bytes / (g_ms * 1e-3) / 1e9, 1),
                                   "frac": round(g_bytes / (g_ms * 1e-3) / 1e9 / peak, 4)},
                        "deposit": {"ms": round(d_ms, 4), "algorithmic_bytes": d_bytes,
                                    "achieved_GBs": round(d_bytes / (d_ms * 1e-3) / 1e9, 1),
                                    "frac": round(d_bytes / (d_ms * 1e-3) / 1e9 / peak, 4)}},
            "peak": peak, "peak_kind": peak_kind, "gpu_launches": int(launches), "clocks": clk.summary()}
    if not args.no_cpu_baseline:
        # the oracle's FP64 restatement on the host cores, on a bounded sample
        from oracle import oracle as O
        m = min(1 << 21, n)   # about ten seconds of the oracle on the host cores
        sample = pos[:, :m].cpu().numpy()
        phi_h = phi.cpu().numpy()
        g = O.make_grid((cells, cells), (0.5, 0.5), (cells + 0.5, cells + 0.5), (0, 0))
        t0 = time.perf_counter()
        O.bspline_gather(g, order, sample, phi_h, grad=True)
        O.bspline_deposit(g, order, sample, 1.0 / ppc, nodes)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": m / dt, "unit": "particles/s", "cores": os.cpu_count(), "kind": "port",
                                "sample": f"first {m} particles of the workload, gather (OpenMP) + deposit (serial)"}
    return line


def run_c4(args, torch, P, w):
    """Forward and adjoint of the differentiable run, timed with CUDA events."""
    from psum_b200.adjoint import ElectrostaticLoss, ElectrostaticRun
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    gen = torch.Generator(device=dev)
    gen.manual_seed(SEED + 4)
    grid, opts, fixed, backend = periodic_problem(P, w, args.mg_extra)
    pos, vel, n = periodic_initial_state(torch, w, gen, dev)
    L = w["cells"] + 1.0
    steps = 100
    run = ElectrostaticRun(grid, (1, 1), [(-1.0, 1.0, L * L / n, pos)], fixed, opts, w["dt"], steps,
                           checkpoint_every=10, precision=P.MIXED, background=1.0)
    phi_ext = (torch.randn(grid.n_nodes, generator=gen, device=dev, dtype=torch.float64) * 0.01)
    v0 = vel.to(torch.float32)
    times = []
    for rep in range(args.warmup + max(args.steps // 10, 1)):
        v = v0.clone().requires_grad_(True)
        pe = phi_ext.clone().requires_grad_(True)
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record()
        loss = ElectrostaticLoss.apply(run, pe, v)
        e1.record()
        loss.backward()
        e2.record()
        torch.cuda.synchronize()
        if rep >= args.warmup:
            times.append((e0.elapsed_time(e1), e1.elapsed_time(e2)))
    fwd = statistics.median(t[0] for t in times)
    bwd = statistics.median(t[1] for t in times)
    return {"workload": "c4", "metric": "particle-steps/s of the differentiable run (forward; forward + adjoint)",
            "value": n * steps / (fwd * 1e-3), "unit": "particle-steps/s", "n_gpus": 1, "steps": steps,
            "warmup": args.warmup, "ms_forward": fwd, "ms_backward": bwd,
            "value_forward_and_adjoint": n * steps / ((fwd + bwd) * 1e-3), "higher_is_better": True,
            "dtype": "f32 push and adjoint arrays / f64 fields", "data": "synthetic",
            "config": {"workload": w["desc"], "particles": n, "nodes": grid.n_nodes, "dt": w["dt"], "mg": opts,
                       "checkpoint_every": 10},
            "loss": float(loss.detach()), "grad_v_norm": float(v.grad.norm()), "grad_phi_ext_norm": float(pe.grad.norm())}


def run_reference(args, rank):
    """The reference arm: whole steps of the CPU restatement of PSuM's
    algorithm (CpuRun) on all host cores, W untimed and K timed steps, each
    step a bounded sample of the workload (the same plasma on a sub-domain)."""
    if rank != 0:
        return None
    run = CpuRun(CPU_CELLS, args.ppc, SEED)
    for _ in range(args.warmup):
        run.step()
    steps = max(args.steps, 1)
    t0 = time.perf_counter()
    for _ in range(steps):
        run.step()
    dt = time.perf_counter() - t0
    value = run.n_total * steps / dt
    return {"impl": "reference",
            "metric": "particle-steps/s incl. Poisson MG, mixed-prec vs FP64 on GPU at stated error",
            "value": value, "unit": "particle-steps/s", "n_gpus": 1, "steps": steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * dt / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args),
            "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": os.cpu_count(), "kind": "port",
                             "sample": run.describe(steps)},
            "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "PSuM cannot be built here (needs AdaptiveCpp and Eigen 3.4); this is the FP64 CPU "
                    "restatement of its algorithm (oracle/) on all host cores"}


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist
        if args.impl == "ours":
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", rank)))
            tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
            dist = tdist
    if args.impl == "reference":
        line = run_reference(args, rank)
    elif args.workload != "c2":
        line = run_workload(args) if rank == 0 else None
    else:
        line = run_ours(args, rank, world, dist)
    if line is not None:
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
