"""Benchmark of the B200 physics stage: Mcell-steps/s on seeded synthetic worlds.

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                [--config hex4m|fluid1m|softbody|batched256]

One step = one timestep of the per-timestep physics stage over the whole
world (cell map, pair forces, bond forces, Verlet, energy particles,
structural operations).  Default workload: the soft-body-heavy world, 4M
cells in 40k hexagonal 100-cell clusters on a 4096x4096 torus, collision
motion, bond breaking on.  State is larger than L2 (126 MB), so no flush is
needed between steps.  Prints one JSON line (rank 0).

--impl reference times the reference's own implementation of the path on
this machine: the reference ships only a CUDA engine, built from its sources
for sm_100a as oracle/_ref/ref_run and stepped from the same world; without
that binary, the CPU restatement of the same step (oracle, FP32, OpenMP over
all host threads) is timed and reported as a port.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-steps/s"
T0 = time.perf_counter()


def log(msg: str) -> None:
    """progress on stderr (the JSON line is the only stdout output)"""
    print(f"[bench {time.perf_counter() - T0:7.1f}s] {msg}", file=sys.stderr, flush=True)

# Algorithmic bytes per cell-step, phase by phase (compulsory FP32 SoA
# traffic of the reference's dependency-separated phases, neighbour reads
# counted 0 as served from shared memory / L2; b = bonds per cell):
#   P1 hash build 24; P2 pair forces 40; P3 apply forces 24;
#   P4 bond forces #1 20 + 12b; P5 Verlet x 32; P6 bond forces #2 20 + 12b;
#   P7 Verlet v + friction 32  ->  B_cell = 192 + 24b.
PHASE_BYTES = {"P1": lambda b: 24.0, "P2": lambda b: 40.0, "P3": lambda b: 24.0, "P4": lambda b: 20.0 + 12.0 * b,
               "P5": lambda b: 32.0, "P6": lambda b: 20.0 + 12.0 * b, "P7": lambda b: 32.0}


def step_bytes_per_cell(bonds_per_cell: float) -> float:
    """B_cell of the whole step: 192 + 24b"""
    return sum(f(bonds_per_cell) for f in PHASE_BYTES.values())


def algorithmic_bytes(kernel: str, bonds_per_cell: float) -> float:
    """Algorithmic bytes per cell of one launch of `kernel`: the phases it
    carries.  The first bond-force kernel also applies the pair forces, and
    does the Verlet position update in the two steps of three without angle
    forces (the position kernel does it in the third)."""
    b = bonds_per_cell
    if kernel.startswith("kPairsRegion"):
        return PHASE_BYTES["P2"](b)
    return {
        "kApplyBond1": PHASE_BYTES["P3"](b) + PHASE_BYTES["P4"](b) + PHASE_BYTES["P5"](b) * 2.0 / 3.0,
        "kVerletPos": PHASE_BYTES["P5"](b) / 3.0,
        "kBond2": PHASE_BYTES["P6"](b),
        "kVerletVel": PHASE_BYTES["P7"](b),
    }.get(kernel, 0.0)


def layout_bytes(kernel: str) -> float:
    """Bytes per cell one launch moves with this engine's data layout (each
    array read or written for the cell counted once: the staged pair record
    is 32 B, a bond row 24 B, rest lengths 24 B, ...): the traffic to expect
    from the layout, as opposed to the algorithmic minimum above."""
    if kernel.startswith("kPairsRegion"):
        return 80.0
    return {"kApplyBond1": 104.0 + 16.0 / 3.0, "kBond2": 80.0, "kVerletPos": 58.0 / 3.0, "kVerletVel": 67.0,
            "kBin": 26.0}.get(kernel, 0.0)


def load_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region"""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


def build_workload(config: str, rank: int = 0):
    from alien_b200 import params as P
    from alien_b200 import worldgen

    seed = 1000 * rank
    if config == "hex4m":
        data, world = worldgen.hex_world(seed=seed)
        prm = P.benchmark_parameters(P.MOTION_COLLISION)
        desc = "soft-body heavy: 4096x4096 torus, 4M cells in 40k hexagonal 100-cell clusters, collisions + bond breaking"
    elif config == "hex1m":
        data, world = worldgen.hex_world(seed=seed, world=(2048, 2048), clusters=10000)
        prm = P.benchmark_parameters(P.MOTION_COLLISION)
        desc = "soft-body, profiling size: 2048x2048 torus, 1M cells in 10k hexagonal 100-cell clusters"
    elif config == "neuron1m":
        import numpy as np
        data, world = worldgen.hex_world(seed=seed, world=(2048, 2048), clusters=10000)
        rng = np.random.default_rng(seed + 1)
        chosen = np.nonzero(rng.random(10000) < 1.0 / 3.0)[0]
        cells = (chosen[:, None] * 100 + np.arange(100)[None, :]).ravel()
        data = worldgen.add_neurons(data, seed + 2, fraction=1.0, cells=cells)
        prm = P.benchmark_parameters(P.MOTION_COLLISION)
        desc = ("soft-body with neurons: hex1m with a third of the clusters made of neuron cells "
                "(8x8 weights ~ N(0, 0.5), biases ~ N(0, 0.1))")
    elif config == "fluid1m":
        data, world = worldgen.fluid_world(seed=seed)
        prm = P.benchmark_parameters(P.MOTION_FLUID)
        desc = "SPH fluid stress: 2048x2048 torus, 1M unbonded cells, density 0.24, velocity sigma 0.5"
    elif config == "softbody":
        data, world = worldgen.soft_body_world(seed=seed)
        prm = P.benchmark_parameters(P.MOTION_FLUID)
        desc = "plain small: 512x512 torus, 200 10x10 lattice clusters (20k cells) + 20k energy particles"
    else:
        raise ValueError(config)
    return data, world, prm, desc


def pin(arr):
    """page-lock a numpy buffer for the host<->device copies of the e2e leg"""
    import torch
    if arr.nbytes == 0:
        return None
    rc = torch.cuda.cudart().cudaHostRegister(arr.ctypes.data, arr.nbytes, 0)
    return arr.ctypes.data if int(rc) == 0 else None


def unpin(ptr):
    import torch
    if ptr:
        torch.cuda.cudart().cudaHostUnregister(ptr)


def cpu_baseline(data, world, prm, budget_s: float = 20.0, max_steps: int = 1000, precision: str = "f32"):
    """The CPU restatement (FP32, OpenMP) stepping the same world: a bounded
    sample of about ``budget_s`` seconds."""
    from oracle.oracle import OracleSimulation, library

    threads = library(precision).oracle_num_threads()
    log(f"cpu baseline: {threads} threads")
    sim = OracleSimulation(world, prm, 0, precision=precision)
    sim.set_simulation_data(data)
    t0 = time.perf_counter()
    sim.calc_timesteps(1)  # warm-up step
    first = time.perf_counter() - t0
    steps = max(1, min(max_steps, int(budget_s / max(first, 1e-6))))
    log(f"cpu baseline: first step {first:.2f} s, timing {steps} steps")
    t0 = time.perf_counter()
    sim.calc_timesteps(steps)
    dt = time.perf_counter() - t0
    sim.close()
    value = data.num_cells * steps / dt / 1e6
    return {"value": value, "unit": METRIC, "cores": threads, "kind": "port",
            "sample": f"{steps} steps of the same world after 1 warm-up step ({dt:.1f} s, {threads} threads)"}, steps, dt


def run_reference(args, config, rank, world_size):
    """--impl reference: the reference path timed on this machine.

    The reference's path is its CUDA engine (_SimulationCudaFacade::
    calcTimestep, source/EngineGpuKernels/SimulationCudaFacade.cu:128-160),
    built from the reference sources for sm_100a as oracle/_ref/ref_run and
    driven through its own facade from the identical DataTO: W warm-up steps,
    then K steps in one calcTimestep(K, false) call timed by wall clock (the
    facade synchronises after every step).  Without that binary (or a GPU),
    the CPU restatement of the same step is timed instead."""
    if rank != 0:
        return 0
    from oracle import refrun

    if config == "batched256":
        return run_reference_batched(args, refrun)
    # The reference engine holds at most about 1.83M cells in one world (its
    # dynamic-memory bound in SimulationData::resizeObjects,
    # SimulationData.cu:93, is an int that overflows for larger cell
    # arrays); the 4M-cell world is timed on its 1M-cell quarter, which has
    # the same density, cluster shape and velocity distribution.
    sample_config = {"hex4m": "hex1m"}.get(config, config)
    data, world, prm, desc = build_workload(sample_config)

    gpu = False
    try:
        import torch
        gpu = torch.cuda.is_available()
    except ImportError:
        pass
    if refrun.available() and gpu:
        log(f"reference CUDA engine: {args.warmup} warm-up + {args.steps} timed steps")
        _, seconds, _ = refrun.run(data, world, prm, steps=args.steps, warmup=args.warmup, timeout=1500)
        value = data.num_cells * args.steps / seconds / 1e6
        line = {
            "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * seconds / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": config, "sample_workload": sample_config, "description": desc,
                       "cells": data.num_cells},
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": 1, "kind": "reference",
                             "sample": f"the reference CUDA engine on cuda:0 (one host thread driving it), "
                                       f"{sample_config} ({data.num_cells} cells): "
                                       f"{args.steps} steps after {args.warmup} warm-up steps"},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference engine (source/EngineGpuKernels, all units) compiled for sm_100a with its own flags; "
                    "timed around _SimulationCudaFacade::calcTimestep(K, false), which synchronises every step",
        }
        print(json.dumps(line))
        return 0
    base, steps, dt = cpu_baseline(data, world, prm, budget_s=min(120.0, 5.0 + 2.0 * args.steps))
    line = {
        "impl": "reference", "metric": METRIC, "value": base["value"], "unit": METRIC, "n_gpus": 0,
        "steps": steps, "warmup": 1, "ms_per_step": 1000.0 * dt / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": config, "description": desc, "cells": data.num_cells},
        "cpu_baseline": base,
        "e2e": {"value": base["value"], "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference CUDA engine not built here; this is the CPU restatement of the same step "
                "(oracle, FP32, OpenMP)",
    }
    print(json.dumps(line))
    return 0


def run_reference_batched(args, refrun, sample: int = 32):
    """the reference engine steps worlds of the 256-world batch one after
    another (it holds one world per facade); timed on the first ``sample``
    worlds, the same worlds as rank 0 of the batched arm"""
    from alien_b200 import params as P
    from alien_b200 import worldgen

    sizes = worldgen.batched_sizes(seed=0, count=256)[:sample]
    cells, seconds = 0, 0.0
    for i, n in enumerate(sizes):
        d, w = worldgen.mixed_world(seed=i, num_cells=int(n))
        _, dt, _ = refrun.run(d, w, P.benchmark_parameters(P.MOTION_FLUID), steps=args.steps, warmup=args.warmup)
        cells += d.num_cells
        seconds += dt
    value = cells * args.steps / seconds / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * seconds / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "batched256", "worlds_timed": sample, "cells": cells},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": 1, "kind": "reference",
                         "sample": f"the reference CUDA engine stepping the first {sample} of the 256 worlds one "
                                   f"after another, {args.steps} steps each after {args.warmup} warm-up steps"},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_batched(args, rank, world_size):
    """256 worlds, log-uniform 1k-200k cells: one arena stepped together vs
    the plain engine stepping the same worlds one after another.

    ``--partition replica`` (default): every rank steps its own 256 worlds
    (weak scaling).  ``--partition global``: the 256 worlds of rank 0 are
    split across the ranks by cell count (strong scaling)."""
    from alien_b200 import params as P
    from alien_b200 import worldgen
    from alien_b200.facade import BatchSimulation, SimulationFacade
    from alien_b200.replicas import partition_worlds

    if args.partition == "global":
        sizes = worldgen.batched_sizes(seed=0, count=256)
        mine = partition_worlds(sizes, world_size)[rank]
        seeds = mine
    else:
        sizes = worldgen.batched_sizes(seed=rank, count=256)
        mine = range(len(sizes))
        seeds = [10_000 * rank + i for i in mine]
    worlds = []
    for i, sd in zip(mine, seeds):
        d, w = worldgen.mixed_world(seed=sd, num_cells=int(sizes[i]))
        worlds.append((d, w, P.benchmark_parameters(P.MOTION_FLUID)))
    total = sum(d.num_cells for d, _, _ in worlds)
    batch = BatchSimulation(worlds)
    batch.calc_timesteps(args.warmup)
    launches0 = batch.kernel_launches()
    with ClockSampler(int(os.environ.get("LOCAL_RANK", 0))) as clk:
        ms = batch.time_timesteps(args.steps)
    launches = batch.kernel_launches() - launches0
    batch.close()
    # plain: each world its own facade, stepped sequentially (same step count)
    plain_steps = max(3, args.steps // 10)
    sims = []
    for d, w, p in worlds:
        s = SimulationFacade()
        s.new_simulation(0, w, p)
        s.set_simulation_data(d)
        s.calc_timesteps(1)
        sims.append(s)
    t_plain = 0.0
    for s in sims:
        t_plain += s.time_timesteps(plain_steps)
    for s in sims:
        s.close_simulation()
    plain_value = total * plain_steps / (t_plain / 1000.0) / 1e6
    value = total * args.steps / (ms / 1000.0) / 1e6
    return {"value": value, "ms": ms, "launches": launches, "clocks": clk.summary(), "total": total,
            "plain_value": plain_value, "plain_ms_per_step": t_plain / plain_steps}


def run_serving(args, rank):
    """Poisson arrivals of simulation requests (worlds of log-uniform
    5k-500k cells built as the batched worlds, log-uniform 100-5000 steps)
    admitted against an HBM budget and stepped together by the continuous-
    batching loop (alien_b200.serving).  The request worlds come from a pool
    built before the run, so world generation on the host stays out of the
    measured loop."""
    import numpy as np
    from alien_b200 import params as P
    from alien_b200 import serving, worldgen

    rng = np.random.default_rng(1000 + rank)
    sizes = np.exp(rng.uniform(math.log(5_000), math.log(500_000), args.pool)).astype(int)
    pool = []
    for i, n in enumerate(sizes):
        d, w = worldgen.mixed_world(seed=100_000 * rank + i, num_cells=int(n))
        # a third of the lattice clusters (the first cells, 100 per cluster)
        # are made of neuron cells
        n_clusters = int(np.sum(d.cells["numConnections"] > 0) // 100)
        chosen = np.nonzero(rng.random(n_clusters) < 1.0 / 3.0)[0]
        d = worldgen.add_neurons(d, 100_000 * rank + i, fraction=1.0,
                                 cells=(chosen[:, None] * 100 + np.arange(100)[None, :]).ravel())
        pool.append((d, w))
    # request data arrives in page-locked host buffers, as a server would keep them
    pins = [pin(d._cells) for d, _ in pool]
    log(f"serving: pool of {len(pool)} worlds, {sum(d.num_cells for d, _ in pool)} cells")
    prm = P.benchmark_parameters(P.MOTION_FLUID)

    def make(rid, r):
        d, w = pool[int(r.integers(len(pool)))]
        steps = int(math.exp(r.uniform(math.log(100), math.log(5000))))
        return serving.Request(rid, d, w, prm, steps)

    with ClockSampler(int(os.environ.get("LOCAL_RANK", 0))) as clk:
        out = serving.run_poisson(make, rate_per_s=args.rate, duration_s=args.duration,
                                  hbm_budget_bytes=int(args.hbm_budget_gb * 1e9), seed=rank, drain=False,
                                  steps_per_tick=args.steps_per_tick, admit_interval=args.admit_interval)
    out["clocks"] = clk.summary()
    for p in pins:
        unpin(p)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="hex4m",
                    choices=["hex4m", "hex1m", "neuron1m", "fluid1m", "softbody", "batched256", "serving"])
    ap.add_argument("--duration", type=float, default=60.0, help="serving: seconds of arrivals")
    ap.add_argument("--rate", type=float, default=20.0, help="serving: mean requests per second")
    ap.add_argument("--pool", type=int, default=32, help="serving: distinct request worlds")
    ap.add_argument("--hbm-budget-gb", type=float, default=150.0, help="serving: admission budget")
    ap.add_argument("--steps-per-tick", type=int, default=8, help="serving: steps of every cohort per loop tick")
    ap.add_argument("--admit-interval", type=float, default=0.0,
                    help="serving: seconds between admission waves while cohorts run")
    ap.add_argument("--partition", default="replica", choices=["replica", "global"],
                    help="batched256: each rank its own 256 worlds, or the 256 worlds split across ranks")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-same-workload", action="store_true",
                    help="hex4m: skip timing the 1M-cell world that the reference arm runs")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", 0))
    world_size = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        return run_reference(args, args.config, rank, world_size)

    import torch

    from alien_b200 import _lib
    from alien_b200.facade import SimulationFacade
    from alien_b200.replicas import Replicas

    reps = Replicas()
    _lib.select_device(local_rank)
    barrier, max_over_ranks, sum_over_ranks = reps.barrier, reps.max, reps.sum

    peak, peak_kind = load_peak()
    if args.config == "serving":
        r = run_serving(args, rank)
        agg = sum_over_ranks(r["cell_steps"]) / max_over_ranks(r["wall_s"]) / 1e6
        if rank == 0:
            line = {
                "metric": METRIC, "value": agg, "unit": METRIC, "n_gpus": world_size, "steps": r["ticks"],
                "warmup": 0, "ms_per_step": r["p50_step_ms"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": "serving", "rate_per_s": args.rate, "duration_s": args.duration,
                           "steps_per_tick": args.steps_per_tick, "admit_interval_s": args.admit_interval,
                           "hbm_budget_gb": args.hbm_budget_gb, "pool_worlds": args.pool,
                           "description": "Poisson arrivals, worlds of log-uniform 5k-500k cells (half fluid, half "
                                          "10x10 lattices, a third of the lattices neuron cells), log-uniform "
                                          "100-5000 steps, continuous batching in one live arena"},
                "p50_step_ms": r["p50_step_ms"], "p99_step_ms": r["p99_step_ms"],
                "admission_wait_s": {"p50": r["p50_admission_wait_s"], "p99": r["p99_admission_wait_s"]},
                "requests": {"submitted": r["requests_submitted"], "finished": r["requests_finished"],
                             "waiting": r["requests_waiting"], "resident": r["requests_resident"]},
                "admission_wave_ms_p50": r["p50_admission_wave_ms"],
                "host_ms": {k: r[k] for k in ("p99_admission_wave_ms", "p50_admit_call_ms", "p99_admit_call_ms",
                                              "p50_sync_ms", "p50_evict_ms")},
                "admissions": r["admissions"], "capacity_events": r["capacity_events"],
                "arena": {"bytes": r["arena_bytes"], "cell_slots": r["arena_cell_slots"],
                          "note": "one live arena: worlds admitted into and evicted from it while the others step"},
                "wall_s": r["wall_s"], "clocks": r["clocks"],
            }
            print(json.dumps(line))
        reps.close()
        return 0
    if args.config == "batched256":
        r = run_batched(args, rank, world_size)
        ms = max_over_ranks(r["ms"])
        total = sum_over_ranks(r["total"])
        if rank == 0:
            line = {
                "metric": METRIC, "value": total * args.steps / (ms / 1000.0) / 1e6, "unit": METRIC,
                "n_gpus": world_size, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "strong" if args.partition == "global" else "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": "batched256", "worlds": 256, "cells": int(total), "partition": args.partition,
                           "parallelism": f"worlds split across {world_size} GPUs by cell count"
                           if args.partition == "global" else f"replicas x{world_size}",
                           "description": "256 worlds, log-uniform 1k-200k cells, density 0.2, half fluid cells and half 10x10 lattices",
                           "l2": "state larger than L2, no flush"},
                "batched_vs_plain": r["value"] / r["plain_value"],
                "plain": {"value": r["plain_value"], "ms_per_step": r["plain_ms_per_step"]},
                "clocks": r["clocks"], "gpu_launches": r["launches"],
            }
            print(json.dumps(line))
        reps.close()
        return 0

    log(f"building workload {args.config}")
    data, world, prm, desc = build_workload(args.config, rank)
    n_cells = data.num_cells
    log(f"workload: {n_cells} cells, {data.num_particles} particles")
    sim = SimulationFacade()
    sim.new_simulation(0, world, prm)
    sim.set_simulation_data(data)
    log("set_simulation_data done; warm-up")
    sim.calc_timesteps(args.warmup)
    stats0 = sim.get_raw_statistics()
    log("timed region")
    launches0 = sim.kernel_launches()
    slots0 = sim.get_array_sizes().particleArraySize
    barrier()
    with ClockSampler(local_rank) as clk:
        ms = sim.time_timesteps(args.steps)
    barrier()
    launches = sim.kernel_launches() - launches0
    stats1 = sim.get_raw_statistics()
    # particle storage grows inside time_timesteps only when a step's new
    # particles did not fit; the world then halted and its missed steps ran
    # after the timed region, so a line with growth would have timed less work
    storage_grew = sim.get_array_sizes().particleArraySize != slots0
    if storage_grew:
        log("WARNING: particle storage grew during the timed region (a world halted): the line is not valid")
    lc = sim.launch_config()
    launch_cfg = {"pair_region_tiles": {"fluid": list(lc.regionTiles[0]), "collision": list(lc.regionTiles[1])},
                  "autotuned": bool(lc.tuned),
                  "tuned_ms_by_region": {m: {f"{lc.candidates[i][k][0]}x{lc.candidates[i][k][1]}": round(lc.tunedMs[i][k], 4)
                                             for k in range(_lib.REGION_CHOICES)} for i, m in enumerate(("fluid", "collision"))}}
    ms = max_over_ranks(ms)
    cells_mean = 0.5 * (stats0.numCells + stats1.numCells)
    total_cells = sum_over_ranks(cells_mean)
    value = total_cells * args.steps / (ms / 1000.0) / 1e6

    log(f"timed region: {ms / args.steps:.3f} ms/step")
    # per-step distribution: each of min(K, 200) further steps between its
    # own pair of CUDA events (a wait between steps, so not the throughput)
    import numpy as np

    step_samples = [sim.time_timesteps(1) for _ in range(min(args.steps, 200))]
    step_p50, step_p99 = (float(np.percentile(step_samples, q)) for q in (50, 99))
    # per-kernel CUDA-event breakdown over a second stretch of the same run
    timed_steps = max(3, min(args.steps, 50))
    kernel_ms = sim.timed_timesteps(timed_steps)
    bonds = stats1.numConnections / max(1, stats1.numCells)
    dominant = max((k for k in kernel_ms if algorithmic_bytes(k, bonds) > 0), key=lambda k: kernel_ms[k])
    per_launch_ms = kernel_ms[dominant] / timed_steps
    alg_bytes = algorithmic_bytes(dominant, bonds) * stats1.numCells
    achieved = alg_bytes / (per_launch_ms / 1000.0) / 1e9
    # every force / integration kernel against the same accounting, and the
    # whole step at B_cell = 192 + 24b
    kernel_roofline = {}
    for k, total_ms in kernel_ms.items():
        ab = algorithmic_bytes(k, bonds)
        if ab > 0:
            gbs = ab * stats1.numCells / (total_ms / timed_steps / 1000.0) / 1e9
            kernel_roofline[k] = {"bytes_per_cell": round(ab, 2), "ms": total_ms / timed_steps, "achieved_gbs": gbs,
                                  "frac": gbs / peak}
    step_gbs = step_bytes_per_cell(bonds) * stats1.numCells / (ms / args.steps / 1000.0) / 1e9
    # DRAM bytes of one launch of the dominant kernel, from a one-kernel ncu
    # capture of this workload (profiles/<kernel>_<workload>_traffic.json)
    traffic = None
    tpath = os.path.join(ROOT, "profiles", f"{dominant.split('<')[0]}_{args.config}_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tj = json.load(f)
        if tj.get("workload") == args.config and tj.get("kernel") == dominant:
            traffic = tj.get("bytes_per_launch")

    # end to end through the C ABI with host buffers: H2D of the world,
    # every step calc_timesteps(1) + a statistics read-back, D2H of the world
    log("kernel breakdown done")
    e2e = None
    if not args.no_e2e:
        pins = [pin(data._cells), pin(data._particles)]
        sizes = None
        sim2 = SimulationFacade()
        sim2.new_simulation(0, world, prm)
        sim2.set_simulation_data(data)
        out = sim2.get_simulation_data()
        out_pins = [pin(out._cells), pin(out._particles)]
        e2e_steps = args.steps
        barrier()
        t0 = time.perf_counter()
        sim2.set_simulation_data(data)
        t_set = time.perf_counter()
        for _ in range(e2e_steps):
            sim2.calc_timesteps(1)
            sim2.get_raw_statistics()
        t_steps = time.perf_counter()
        sim2.get_simulation_data(out=out)
        barrier()
        t_end = time.perf_counter()
        t_e2e = max_over_ranks(t_end - t0)
        log(f"e2e: set_simulation_data {1e3 * (t_set - t0):.1f} ms, {e2e_steps} x (calc_timesteps(1) + "
            f"get_raw_statistics) {1e3 * (t_steps - t_set) / e2e_steps:.3f} ms each, get_simulation_data "
            f"{1e3 * (t_end - t_steps):.1f} ms")
        sim2.close_simulation()
        for p in pins + out_pins:
            unpin(p)
        h2d = data.nbytes() / e2e_steps
        d2h = (out.nbytes() + 112 * e2e_steps) / e2e_steps
        e2e = {"value": sum_over_ranks(n_cells) * e2e_steps / t_e2e / 1e6, "unit": METRIC,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "note": "set_simulation_data + per step (calc_timesteps(1) + get_raw_statistics) + get_simulation_data, pinned host buffers"}

    log("e2e done")
    sim.close_simulation()
    # the 4M-cell world does not fit the reference engine (its memory bound
    # overflows above about 1.83M cells), so the reference arm times the
    # 1M-cell quarter of the same workload; the same process times this
    # engine on that world too, device-resident and end to end
    same = None
    if args.config == "hex4m" and not args.no_same_workload:
        same = time_same_workload(args, rank, barrier, max_over_ranks, sum_over_ranks)
    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        cpu, _, _ = cpu_baseline(data, world, prm)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world_size, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak" if world_size > 1 else "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": args.config, "description": desc, "cells": n_cells,
                       "world": list(world), "bonds_per_cell": round(bonds, 3),
                       "parallelism": f"replicas x{world_size}" if world_size > 1 else "single world",
                       "l2": "state larger than L2 (126 MB), no flush between steps"},
            "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "algorithmic_bytes_per_cell": algorithmic_bytes(dominant, bonds),
                         "layout_bytes_per_launch": layout_bytes(dominant) * stats1.numCells,
                         "launch_ms": per_launch_ms,
                         "note": "achieved = algorithmic bytes per launch (phase accounting, P2 = 40 B/cell) / "
                                 "CUDA-event launch time; layout bytes = what this engine's arrays move per launch"},
            "kernel_roofline": kernel_roofline,
            "step_roofline": {"bytes_per_cell": step_bytes_per_cell(bonds), "achieved_gbs": step_gbs,
                              "frac": step_gbs / peak, "note": "whole step, B_cell = 192 + 24b"},
            "same_workload_as_reference": same,
            "launch_config": launch_cfg,
            "kernel_ms_per_step": {k: v / timed_steps for k, v in kernel_ms.items()},
            "step_ms": {"p50": step_p50, "p99": step_p99, "samples": len(step_samples),
                        "note": "single steps between CUDA events, after the timed region"},
            "clocks": clk.summary(),
            "gpu_launches": launches,
            "particle_storage_grew_in_timed_region": storage_grew,
            "e2e": e2e,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    reps.close()
    return 0


def time_same_workload(args, rank, barrier, max_over_ranks, sum_over_ranks):
    """hex1m (the reference arm's world): device-resident steps and the same
    end-to-end loop as the headline line, K steps after W warm-up steps"""
    from alien_b200.facade import SimulationFacade

    log("same-workload leg: hex1m")
    data, world, prm, desc = build_workload("hex1m", rank)
    sim = SimulationFacade()
    sim.new_simulation(0, world, prm)
    sim.set_simulation_data(data)
    sim.calc_timesteps(args.warmup)
    barrier()
    ms = max_over_ranks(sim.time_timesteps(args.steps))
    barrier()
    sim.close_simulation()
    n = data.num_cells
    out = {"workload": "hex1m", "description": desc, "cells": n,
           "value": sum_over_ranks(n) * args.steps / (ms / 1000.0) / 1e6, "unit": METRIC,
           "ms_per_step": ms / args.steps}
    if not args.no_e2e:
        pins = [pin(data._cells), pin(data._particles)]
        sim2 = SimulationFacade()
        sim2.new_simulation(0, world, prm)
        sim2.set_simulation_data(data)
        res = sim2.get_simulation_data()
        out_pins = [pin(res._cells), pin(res._particles)]
        barrier()
        t0 = time.perf_counter()
        sim2.set_simulation_data(data)
        for _ in range(args.steps):
            sim2.calc_timesteps(1)
            sim2.get_raw_statistics()
        sim2.get_simulation_data(out=res)
        barrier()
        t_e2e = max_over_ranks(time.perf_counter() - t0)
        sim2.close_simulation()
        for p in pins + out_pins:
            unpin(p)
        out["e2e"] = {"value": sum_over_ranks(n) * args.steps / t_e2e / 1e6, "unit": METRIC,
                      "h2d_bytes_per_step": data.nbytes() / args.steps,
                      "d2h_bytes_per_step": (res.nbytes() + 112 * args.steps) / args.steps}
    log(f"same-workload leg: {ms / args.steps:.3f} ms/step")
    return out


if __name__ == "__main__":
    sys.exit(main())
