"""Benchmark of the collision hot path: cell-steps/s of the hard model.

Workload (default): config 2 -- one colony grown by this library from a
single cell to radius 260 in config 2's mixed precision (the reference's
largest published run: R = 260, about 3e5 cells), stored as the start state
proliferatingcellcollectives-idp_b200/data/colony_r260_seed0.npz (made by
`bench.py --grow --radius 260 --precision mixed --save ...`, in two pieces
joined by --checkpoint / --resume).  A step is one
full simulator step on it through the C ABI -- divide, x-sort renumbering,
the ReLCP loop of contact detection and BBPGD solves, motion, growth and
the CFL time-step adaptation (capped at 1e-3) -- in config 2's mixed
precision; the same steps in plain FP64 are reported beside it.  value = sum
of cells over the K timed steps / device time (CUDA events on the library's
stream), summed over ranks; each rank runs its own colony (replicas, no
collective on the data path: weak scaling).  Configs 0 and 1 (hard and soft
colonies grown from one cell to R = 20) run as whole runs after it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference simulator's own C++ code (compiled in
place against single-rank PETSc/MPI stand-ins, oracle/_ref/libpccref_fast.so,
release flags, one thread) on the same colony state.  A full reference step
there takes minutes, so each of its steps is a bounded sample: the
reference's own solver call with its BBPGD capped at a few iterations, whose
time (detection, assembly, iterations) is scaled to a whole step with the
ReLCP phases and BBPGD iterations per step that the same colony needs.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
import pcc_pkg  # noqa: E402

pcc_pkg.load_package()
from pcc_b200 import abi, synth  # noqa: E402

METRIC = "cell-steps/s to R_end; served colonies/s, p50/p99 vs plain GPU at same LCP tol"
UNIT = "cell-steps/s"
RADIUS = 260.0
SNAPSHOT = ROOT / "proliferatingcellcollectives-idp_b200" / "data" / "colony_r260_seed0.npz"
REF_SAMPLE_ITERS = (10, 30)  # BBPGD iterations of the reference's bounded samples
REF_BUDGET_S = 150.0  # wall-clock bound of the reference arm's samples
# algorithmic bytes of one BBPGD iteration per constraint and per cell (the
# mixed-precision form halves the floating-point operand terms)
ALGO_BYTES = {"fp64": (312.0, 288.0), "mixed": (192.0, 144.0)}


def colony_params(**over) -> abi.Params:
    kw = dict(dt=3e-4, fixed_dt=0, dt_cap=1e-3, mode=abi.MODE_HARD, ghost_mode=abi.GHOSTS_SINGLE_RANK, seed=0)
    kw.update(over)
    return abi.default_params(**kw)


def make_colony(radius: float, seed: int) -> dict:
    return synth.dense_colony(radius, seed=seed, lane_gap=0.0, end_gap=0.0)


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "fallback": True}


def traffic_ratio(profile: str) -> float | None:
    """DRAM bytes / algorithmic bytes of a BBPGD kernel from its committed ncu
    summary (profiles/<profile>.md, line 'dram_to_algorithmic: <ratio>')."""
    f = ROOT / "profiles" / f"{profile}.md"
    if f.exists():
        m = re.search(r"dram_to_algorithmic:\s*([0-9.eE+-]+)", f.read_text())
        if m:
            return float(m.group(1))
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_backend() -> str:
    """nccl for the replicas on GPUs; gloo (PCC_BENCH_BACKEND=gloo) for the
    CPU test of the launch and aggregation path."""
    return os.environ.get("PCC_BENCH_BACKEND", "nccl")


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if dist_backend() == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(dist_backend(), timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def spawn_ranks(n: int) -> int:
    """`bench.py --gpus N` without a launcher: starts N copies of this command,
    one rank per GPU (RANK, LOCAL_RANK, WORLD_SIZE and the rendezvous on
    127.0.0.1 in the environment), passes rank 0's output through and returns
    the first non-zero exit status."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    procs = []
    for r in range(n):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(n), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, str(Path(__file__).resolve()), *sys.argv[1:]], env=env,
                                      stdout=None if r == 0 else subprocess.DEVNULL))
    rcs = [pr.wait() for pr in procs]
    return next((rc for rc in rcs if rc), 0)


def _tensor_device() -> str:
    return "cuda" if dist_backend() == "nccl" else "cpu"


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def reduce_max(world: int, v: float) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=_tensor_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(world: int, v: float) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=_tensor_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def run_replica_selftest(args):
    """The replica launch and aggregation without a GPU (the CPU test of the
    --gpus N path): each rank steps its own small colony on the plain-C
    oracle, takes a stand-in time of 100 + 50 * rank ms, and rank 0 prints the
    whole-job line the GPU run would: cell-steps summed over ranks, time the
    max over ranks."""
    world, rank, _ = dist_setup()
    sys.path.insert(0, str(ROOT / "tests"))
    from oracles import OracleColony
    p = abi.default_params(dt=1e-3, fixed_dt=1, seed=rank)
    o = OracleColony(p)
    o.set_cells(abi.seed_cell(rank))
    cells = float(sum(o.step()["n_cells"] for _ in range(max(args.steps, 1))))
    ms = 100.0 + 50.0 * rank
    ms_max = reduce_max(world, ms)
    total = reduce_sum(world, cells)
    if rank == 0:
        print(json.dumps({"n_gpus": world, "value": total / (ms_max / 1e3), "ms_max": ms_max,
                          "cell_steps": total, "rank0_cell_steps": cells}), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def aggregate(cells_per_rank: list[float], ms_per_rank: list[float]) -> tuple[float, float]:
    """Whole-job throughput: all ranks' cell-steps over the slowest rank's time."""
    t = max(ms_per_rank)
    return sum(cells_per_rank) / (t / 1e3), t


def headline_config(n: int, radius: float, world: int, meta: dict) -> dict:
    """The workload description both arms print (identical for the same colony)."""
    return {"workload": f"hard model colony steps, grown colony R={radius:.0f} (config 2), mixed precision",
            "cells": int(n), "start_state": meta.get("start_state", SNAPSHOT.name), "tolerance": 1e-3, "dt": "CFL-adaptive, cap 1e-3",
            "ghost_mode": "single_rank", "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (state + constraints > 126 MB per step)"}


def reference_step_model(cells: dict, dt: float, phases: float, iters: float, repeats: int = 1) -> dict:
    """Time of one reference step on `cells`, from bounded samples of the
    reference's own code (release build, one thread): its solver call with
    BBPGD capped at REF_SAMPLE_ITERS iterations (the reference stops there
    with its 'BBPGD did not converge' error); the difference of the two caps
    gives the time per BBPGD iteration, the rest is the detection and
    assembly of a ReLCP phase.  A step is scaled as phases x (detection +
    assembly) + iters x (time per iteration)."""
    sys.path.insert(0, str(ROOT / "tests"))
    from oracles import RefColony
    times = {j: [] for j in REF_SAMPLE_ITERS}
    for _ in range(repeats):
        for j in REF_SAMPLE_ITERS:
            p = colony_params(dt=dt, max_bbpgd_iterations=j)
            col = RefColony(p, fast=True)
            col.set_cells(cells)
            t0 = time.perf_counter()
            try:
                col.solve(dt, 1)
            except RuntimeError:
                pass  # stopped at the iteration cap
            times[j].append(time.perf_counter() - t0)
    t_lo, t_hi = (float(np.median(times[j])) for j in REF_SAMPLE_ITERS)
    j_lo, j_hi = REF_SAMPLE_ITERS
    t_iter = max((t_hi - t_lo) / (j_hi - j_lo), 0.0)
    t_phase = max(t_lo - j_lo * t_iter, 0.0)
    t_step = phases * t_phase + iters * t_iter
    n = len(cells["x"])
    return {"t_iteration_s": t_iter, "t_phase_s": t_phase, "t_step_s": t_step, "cell_steps_per_s": n / t_step,
            "sampled_s": float(sum(sum(v) for v in times.values())), "phases_per_step": phases,
            "bbpgd_iterations_per_step": iters}


def start_state() -> tuple[dict, float, dict]:
    """The grown R = 260 colony, or -- only if its file is missing -- the
    synthetic dense packing of the same radius, labelled as such."""
    if SNAPSHOT.exists():
        return load_snapshot(str(SNAPSHOT))
    cells = make_colony(RADIUS, seed=0)
    return cells, 3e-4, {"radius": RADIUS, "tail_relcp": [2], "tail_bbpgd": [60],
                         "start_state": "synthetic dense packing (grown colony file missing)"}


def run_reference(args):
    world, rank = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cells, dt, meta = start_state()
    n = len(cells["x"])
    # ReLCP phases and BBPGD iterations per step of this colony, as the run that grew it measured them
    phases = float(np.mean(meta["tail_relcp"]))
    iters = float(np.mean(meta["tail_bbpgd"]))
    # each sample is two reference solver calls on the full colony (tens of
    # seconds at R = 260), so warm-up and timed samples stop once REF_BUDGET_S
    # is spent (at least one timed sample); the line says how many ran
    t0 = time.perf_counter()
    for _ in range(min(args.warmup, 1)):
        reference_step_model(cells, dt, phases, iters)
    samples = []
    while len(samples) < max(args.steps, 1) and (not samples or time.perf_counter() - t0 < REF_BUDGET_S):
        samples.append(reference_step_model(cells, dt, phases, iters))
    el = time.perf_counter() - t0
    t_step = float(np.mean([m["t_step_s"] for m in samples]))
    rate = n / t_step
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (colony grown by this library)",
        "config": headline_config(n, meta["radius"], world, meta),
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": f"each step a bounded sample on the same R={meta['radius']:.0f} colony ({n} "
                                   f"cells): the reference's solver call with BBPGD capped at "
                                   f"{REF_SAMPLE_ITERS[0]} and {REF_SAMPLE_ITERS[1]} iterations, scaled to "
                                   f"{phases:.1f} ReLCP phases and {iters:.0f} BBPGD iterations per step (the "
                                   f"colony's own counts); {samples[-1]['t_iteration_s'] * 1e3:.1f} ms per BBPGD "
                                   f"iteration, {samples[-1]['t_phase_s']:.2f} s per phase of detection and "
                                   f"assembly; release build, one rank, one thread; {len(samples)} timed "
                                   f"sample(s) of the {args.steps} asked for, {el:.0f} s in all"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def timed_steps(col, stream, steps: int, verbose: bool = False):
    """K steps of a colony between two CUDA events on its stream."""
    import torch
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    hist = []
    e0.record(stream)
    for _ in range(steps):
        hist.append(col.step())
        if verbose:
            print(json.dumps(hist[-1]), file=sys.stderr, flush=True)
    e1.record(stream)
    e1.synchronize()
    return hist, e0.elapsed_time(e1)


def roofline(prof: dict, precision: str, peaks: dict) -> dict:
    bb_ms = prof["bbpgd_ms"]
    achieved = prof["bbpgd_algo_bytes"] / (bb_ms / 1e3) / 1e9 if bb_ms > 0 else 0.0
    mixed = precision == "mixed"
    ratio = traffic_ratio("k_bbpgd_planar_mixed_frozen_grown_r260" if mixed else "k_bbpgd_planar_frozen_grown_r260")
    launches_bb = max(prof["bbpgd_launches"], 1)
    return {"bound": "hbm", "achieved": achieved, "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
            "frac": achieved / peaks["hbm_gbs"] if peaks.get("hbm_gbs") else None,
            "traffic": ratio * prof["bbpgd_algo_bytes"] / launches_bb if ratio else None,
            "kernel": f"k_bbpgd_planar<{'float' if mixed else 'double'}> (persistent BBPGD)",
            "peak_source": "fallback" if peaks.get("fallback") else "measured"}


def run_ours(args):
    world, rank, local = dist_setup()
    from pcc_b200 import build, device
    if rank == 0:
        build.build()
    barrier(world)
    import torch
    torch.cuda.init()
    cells, dt0, meta = start_state()
    n0 = len(cells["x"])
    peaks = measured_peaks()

    def colony(precision: int):
        p = colony_params(dt=dt0, capacity_hint=int(n0 * 1.2), precision=precision)
        c = device.Colony(p, device=local)
        c.set_cells(cells)
        return c, p, torch.cuda.ExternalStream(c.stream, device=f"cuda:{local}")

    # ---- headline: config 2 in mixed precision
    col, p, stream = colony(abi.PRECISION_MIXED)
    for _ in range(args.warmup):
        col.step()
    errors = precision_errors(device, col, p, local) if rank == 0 else None
    col.profiling(True)
    launches0 = col.launches
    barrier(world)
    with ClockSampler(local) as clk:
        hist, ms = timed_steps(col, stream, args.steps, args.verbose)
    barrier(world)
    launches = col.launches - launches0
    prof = col.profile()
    cells_steps = float(sum(h["n_cells"] for h in hist))
    ms_max = reduce_max(world, ms)
    value = reduce_sum(world, cells_steps) / (ms_max / 1e3)
    iters_step = prof["bbpgd_iterations"] / max(args.steps, 1)
    phases_step = float(np.mean([h["relcp_iterations"] for h in hist])) if hist else 0.0

    # ---- end to end through the C ABI with host buffers: upload the state
    # from pinned host memory, step, read the state back, every step
    n_cap = int(hist[-1]["n_cells"] * 1.3) + 16
    host = {f: torch.empty(n_cap, dtype=torch.float64, pin_memory=True) for f in abi.CELL_FIELDS}
    host["age"] = torch.empty(n_cap, dtype=torch.int32, pin_memory=True)
    host["force"] = torch.empty(6 * n_cap, dtype=torch.float64, pin_memory=True)
    host["velocity"] = torch.empty(6 * n_cap, dtype=torch.float64, pin_memory=True)
    import ctypes as C
    cs = abi.Cells()
    for f in abi.CELL_FIELDS + ("force", "velocity"):
        setattr(cs, f, C.cast(host[f].data_ptr(), C.POINTER(C.c_double)))
    cs.age = C.cast(host["age"].data_ptr(), C.POINTER(C.c_int))

    class Pinned:
        struct = cs
        cap = n_cap

    n = col.download(Pinned)
    per_cell_bytes = 8 * len(abi.CELL_FIELDS) + 4 + 8 * 12
    h2d = d2h = 0
    e2e_cells = 0.0
    barrier(world)
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    e2e_steps = max(1, args.steps)
    for _ in range(e2e_steps):
        col.upload(Pinned, n)
        h2d += n * per_cell_bytes
        st = col.step()
        e2e_cells += st["n_cells"]
        n = col.download(Pinned)
        d2h += n * per_cell_bytes
    t1.record(stream)
    t1.synchronize()
    barrier(world)
    e2e_ms = reduce_max(world, t0.elapsed_time(t1))
    e2e_value = reduce_sum(world, e2e_cells) / (e2e_ms / 1e3)
    col.close()

    # ---- the same steps in plain FP64 (the north star's plain method)
    col64, p64, stream64 = colony(abi.PRECISION_FP64)
    for _ in range(args.warmup):
        col64.step()
    col64.profiling(True)
    barrier(world)
    hist64, ms64 = timed_steps(col64, stream64, args.steps)
    barrier(world)
    prof64 = col64.profile()
    ms64_max = reduce_max(world, ms64)
    value64 = reduce_sum(world, float(sum(h["n_cells"] for h in hist64))) / (ms64_max / 1e3)
    final64 = col64.get_cells() if rank == 0 else None
    col64.close()

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 operands / f64 accumulation",
        "data": "synthetic (colony grown by this library from one cell)",
        "config": headline_config(n0, meta["radius"], world, meta),
        "roofline": roofline(prof, "mixed", peaks),
        "bbpgd_iterations_per_s": prof["bbpgd_iterations"] / (ms / 1e3),
        "bbpgd_iterations_per_step": iters_step, "relcp_phases_per_step": phases_step,
        "bbpgd_iterations_per_step_thesis_r260": 7800,
        "stage_ms": {"bbpgd": prof["bbpgd_ms"], "detect": prof["detect_ms"], "solve": prof["solve_ms"], "total": ms},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d // e2e_steps,
                "d2h_bytes_per_step": d2h // e2e_steps},
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "fp64": {"value": value64, "ms_per_step": ms64_max / args.steps,
                 "bbpgd_iterations_per_step": prof64["bbpgd_iterations"] / max(args.steps, 1),
                 "roofline": roofline(prof64, "fp64", peaks)},
    }
    if final64 is not None:
        line["packing_fraction"] = packing_fraction(final64)
    if errors is not None:
        line["mixed_vs_fp64"] = errors
    if rank == 0 and world == 1 and not args.no_cpu:
        ref = reference_step_model(cells, dt0, phases_step, iters_step)
        line["cpu_baseline"] = {
            "value": ref["cell_steps_per_s"], "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"the reference's solver call (release build, one thread) on the same R={meta['radius']:.0f} "
                      f"colony with BBPGD capped at {REF_SAMPLE_ITERS[0]} and {REF_SAMPLE_ITERS[1]} iterations "
                      f"({ref['sampled_s']:.0f} s): {ref['t_iteration_s'] * 1e3:.1f} ms per BBPGD iteration, "
                      f"{ref['t_phase_s']:.2f} s per ReLCP phase of detection and assembly, scaled to the "
                      f"{phases_step:.1f} phases and {iters_step:.0f} iterations per step of the timed GPU steps",
            "bbpgd_iterations_per_s": 1.0 / ref["t_iteration_s"] if ref["t_iteration_s"] > 0 else None}
    if rank == 0 and not args.no_small:
        line["config0"] = grow_small(device, local, soft=False)
        line["config1"] = grow_small(device, local, soft=True)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def grow_small(device, local: int, soft: bool) -> dict:
    """Configs 0 and 1 as whole runs: one colony grown from a single cell
    (orientation from seed 0) to R = 20 -- hard model, FP64, dt = 1e-3 fixed;
    or soft model, dt = 3e-5, kcc = 4/3 E (E = 1e3, R_eff = 0.125) -- timed
    with CUDA events; for the soft colony also config 1's microbench, the force
    and torque assembly on its final state repeated 1e4 times, with its
    roofline on 104 B per contact and 56 B per cell."""
    import torch
    if soft:
        p = abi.default_params(dt=3e-5, fixed_dt=1, seed=0, mode=abi.MODE_SOFT, kcc=1333.3333333333333)
    else:
        p = abi.default_params(dt=1e-3, fixed_dt=1, seed=0, mode=abi.MODE_HARD)
    col = device.Colony(p, device=local)
    col.set_cells(abi.seed_cell(0))
    stream = torch.cuda.ExternalStream(col.stream, device=f"cuda:{local}")
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0 = time.time()
    e0.record(stream)
    steps, cell_steps, st = col.run(20.0, 10**7)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    out = {"workload": ("soft" if soft else "hard") + " colony grown from one cell to R=20",
           "steps": steps, "cells": st["n_cells"], "cell_steps_per_s": cell_steps / (ms / 1e3),
           "device_s": ms / 1e3, "wall_s": time.time() - w0, "us_per_step": ms * 1e3 / max(steps, 1)}
    if soft:
        reps = 10000
        t = col.soft_forces_frozen(reps)
        m = col.detect(0.0)["sd"].size
        algo = 104.0 * m + 56.0 * st["n_cells"]
        out["frozen_assembly"] = {"repeats": reps, "contacts": m, "us_per_assembly": t * 1e3,
                                  "algo_gbs": algo / (t / 1e3) / 1e9,
                                  "frac_of_hbm": algo / (t / 1e3) / 1e9 / measured_peaks()["hbm_gbs"]}
    col.close()
    return out


def packing_fraction(c: dict) -> float:
    """Cell area (2D spherocylinders) over the area of the colony disk, whose
    radius is the largest distance of a segment end from the origin."""
    d, L = np.asarray(c["diameter"]), np.asarray(c["length"])
    th = 2.0 * np.arctan2(np.asarray(c["q3"]), np.asarray(c["q0"]))
    half = L / 2 - d / 2
    x, y = np.asarray(c["x"]), np.asarray(c["y"])
    ex, ey = half * np.cos(th), half * np.sin(th)
    r = np.sqrt(np.maximum((x + ex) ** 2 + (y + ey) ** 2, (x - ex) ** 2 + (y - ey) ** 2))
    area = np.sum(np.pi * d * d / 4 + d * (L - d))
    return float(area / (np.pi * r.max() ** 2))


def precision_errors(device, col, p, local) -> dict:
    """One solver call from the same state with the FP64 and the mixed-precision
    solver: errors of gamma (phase-0 rows, identical in both), cell forces and
    positions, and the packing fraction, relative to FP64."""
    snap = col.get_cells()
    dt = col.dt
    out = {}
    for name, prec in (("fp64", abi.PRECISION_FP64), ("mixed", abi.PRECISION_MIXED)):
        q = abi.Params.from_buffer_copy(p)
        q.precision = prec
        c = device.Colony(q, device=local)
        c.set_cells(snap)
        st = c.solve(dt, 0)
        out[name] = (st, c.get_cells(), c.constraints())
        c.close()
    (s0, c0, k0), (s1, c1, k1) = out["fp64"], out["mixed"]
    r0 = k0["phase"] == 0
    r1 = k1["phase"] == 0
    g0, g1 = k0["gamma"][r0], k1["gamma"][r1]
    same_rows = bool(r0.sum() == r1.sum() and np.array_equal(k0["gid_i"][r0], k1["gid_i"][r1]))
    f0, f1 = c0["force"], c1["force"]
    return {
        "state": f"after the warm-up steps ({len(snap['x'])} cells), one solver call each",
        "gamma_phase0_max_abs": float(np.max(np.abs(g0 - g1))) if same_rows else None,
        "gamma_phase0_rel": float(np.max(np.abs(g0 - g1)) / max(np.max(np.abs(g0)), 1e-300)) if same_rows else None,
        "force_rel": float(np.max(np.abs(f0 - f1)) / max(np.max(np.abs(f0)), 1e-300)),
        "position_max_abs": float(max(np.max(np.abs(c0[k] - c1[k])) for k in ("x", "y"))),
        "packing_fraction": {"fp64": packing_fraction(c0), "mixed": packing_fraction(c1)},
        "residual": {"fp64": s0["residual"], "mixed": s1["residual"]},
        "max_overlap": {"fp64": s0["max_overlap"], "mixed": s1["max_overlap"]},
        "bbpgd_iterations": {"fp64": s0["bbpgd_iterations"], "mixed": s1["bbpgd_iterations"]},
        "relcp_iterations": {"fp64": s0["relcp_iterations"], "mixed": s1["relcp_iterations"]},
        "tolerance": p.tolerance,
    }


def run_frozen(args):
    """BBPGD microbench on a frozen state: after W warm-up steps, detect the
    phase-0 contacts once and time `--steps` solves of that constraint set
    (the captured launch of the committed ncu summaries)."""
    from pcc_b200 import device
    if args.start == "grown":
        cells, dt0, _ = start_state()
    else:
        cells, dt0 = make_colony(args.radius, seed=0), 3e-4
    prec = abi.PRECISION_MIXED if args.precision == "mixed" else abi.PRECISION_FP64
    # --frozen-tol loosens the BBPGD tolerance of the frozen solves only, which
    # bounds a launch's iterations (for a profiler capture); the traffic of one
    # iteration does not depend on it
    col = device.Colony(colony_params(dt=dt0, capacity_hint=int(len(cells["x"]) * 1.5), precision=prec,
                                      tolerance=args.frozen_tol))
    col.set_cells(cells)
    for _ in range(args.warmup):
        col.step()
    n = col.n_cells
    col.profiling(True)
    it, res, ms = col.bbpgd_frozen(col.dt, max(args.steps, 1))
    prof = col.profile()
    bc, bn = ALGO_BYTES[args.precision]
    m = int(round((prof["bbpgd_algo_bytes"] / max(prof["bbpgd_iterations"], 1) - bn * n) / bc))
    algo = it * (bc * m + bn * n)
    print(json.dumps({"frozen_bbpgd": True, "precision": args.precision, "start": args.start, "radius": args.radius,
                      "tolerance": args.frozen_tol,
                      "cells": n, "constraints": m, "iterations": it, "us_per_iteration": ms * 1e3 / max(it, 1),
                      "residual": res, "ms_per_solve": ms, "algo_bytes_per_solve": algo,
                      "algo_gbs": algo / (ms / 1e3) / 1e9,
                      "frac_of_hbm": algo / (ms / 1e3) / 1e9 / measured_peaks()["hbm_gbs"]}), flush=True)


def run_grow(args):
    """Grows one colony from a single cell (orientation from the seed) to
    --radius with the hard model, CFL-adaptive dt capped at 1e-3 -- the run the
    reference's R = 260 figures come from -- and reports the whole run."""
    import torch
    from pcc_b200 import build, device
    build.build()
    torch.cuda.init()
    prec = abi.PRECISION_MIXED if args.precision == "mixed" else abi.PRECISION_FP64
    done = {"steps": 0, "cell_steps": 0.0, "bbpgd": 0, "device_s": 0.0, "wall_s": 0.0, "segment": 0,
            "stage_ms": {"bbpgd": 0.0, "detect": 0.0, "solve": 0.0}, "marks": []}
    if args.resume:  # an earlier segment of the same run (its --checkpoint file)
        ck = np.load(args.resume, allow_pickle=False)
        done = json.loads(str(ck["run"]))
        done["segment"] += 1
    # a resumed segment draws its division lengths from its own stream (the
    # context's position in the first stream is not part of the saved state)
    p = colony_params(dt=1e-3, precision=prec, capacity_hint=int(4.5 * args.radius ** 2 * 1.2) + 64,
                      seed=args.job_seed + done["segment"])
    col = device.Colony(p)
    if args.resume:
        col.set_cells({k[5:]: ck[k] for k in ck.files if k.startswith("cell_")})
        col.dt = float(ck["dt"])
        col.set_clock(float(ck["sim_time"]), done["steps"])
    else:
        col.set_cells(abi.seed_cell(args.job_seed))
    stream = torch.cuda.ExternalStream(col.stream, device="cuda:0")
    col.profiling(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.time()
    tlast = t0
    steps = bb = 0
    cells = 0.0
    radius = float(ck["radius"]) if args.resume else 0.0
    marks = done["marks"]
    from collections import deque
    tail = deque(maxlen=50)  # solver statistics of the last steps, kept with a saved snapshot
    e0.record(stream)
    st = {}
    while radius < args.radius and time.time() - t0 < args.grow_seconds:
        st = col.step()
        steps += 1
        cells += st["n_cells"]
        bb += st["bbpgd_iterations"]
        radius = st["colony_radius"]
        if not marks or radius >= marks[-1]["radius"] + 20.0:
            marks.append({"radius": radius, "step": done["steps"] + steps, "cells": st["n_cells"],
                          "wall_s": done["wall_s"] + time.time() - t0, "dt": st["dt_used"],
                          "bbpgd_step": st["bbpgd_iterations"]})
        if time.time() - tlast > 10:
            tlast = time.time()
            print(json.dumps({"step": done["steps"] + steps, "radius": radius, "cells": st["n_cells"],
                              "dt": st["dt_used"], "bbpgd": st["bbpgd_iterations"], "wall_s": tlast - t0}),
                  file=sys.stderr, flush=True)
        tail.append(st)
    e1.record(stream)
    e1.synchronize()
    wall = time.time() - t0
    dev_ms = e0.elapsed_time(e1)
    prof = col.profile()
    final = col.get_cells()
    run = {"steps": done["steps"] + steps, "cell_steps": done["cell_steps"] + cells, "bbpgd": done["bbpgd"] + bb,
           "device_s": done["device_s"] + dev_ms / 1e3, "wall_s": done["wall_s"] + wall, "segment": done["segment"],
           "stage_ms": {"bbpgd": done["stage_ms"]["bbpgd"] + prof["bbpgd_ms"],
                        "detect": done["stage_ms"]["detect"] + prof["detect_ms"],
                        "solve": done["stage_ms"]["solve"] + prof["solve_ms"]},
           "marks": marks}
    if args.checkpoint:  # the exact state a next step reads (forces and velocities are recomputed), for --resume
        np.savez_compressed(args.checkpoint, dt=np.float64(col.dt), sim_time=np.float64(st.get("sim_time", 0.0)),
                            radius=np.float64(radius), run=np.array(json.dumps(run)),
                            **{"cell_" + k: np.asarray(v) for k, v in final.items()
                               if k not in ("force", "velocity", "num_constraints")})
    if args.save:
        save_snapshot(args.save, final, col.dt, run["steps"], st, tail, args.job_seed)
    print(json.dumps({
        "grow": True, "precision": args.precision, "radius_target": args.radius, "radius": radius,
        "reached": radius >= args.radius, "segments": run["segment"] + 1, "steps": run["steps"],
        "cells": int(st.get("n_cells", 1)), "cell_steps": run["cell_steps"], "wall_s": run["wall_s"],
        "device_s": run["device_s"], "cell_steps_per_s": run["cell_steps"] / run["device_s"],
        "bbpgd_iterations": run["bbpgd"], "bbpgd_iterations_per_s": run["bbpgd"] / run["device_s"],
        "stage_ms": run["stage_ms"], "packing_fraction": packing_fraction(final), "sim_time": st.get("sim_time"),
        "marks": marks, "segment_steps": steps, "segment_device_s": dev_ms / 1e3,
    }), flush=True)


def save_snapshot(path: str, cells: dict, dt: float, steps: int, last: dict, tail: list, seed: int):
    """A grown colony as the benchmark's starting state: centres, orientation
    angle and length as float32 (the start of a step tolerates the rounding:
    it moves cells by < 3e-5, far below the solver tolerance), birth length and
    diameter as float32, age as int32, with the run that made it."""
    th = 2.0 * np.arctan2(np.asarray(cells["q3"]), np.asarray(cells["q0"]))
    np.savez_compressed(path, x=np.asarray(cells["x"], np.float32), y=np.asarray(cells["y"], np.float32),
                        theta=th.astype(np.float32), length=np.asarray(cells["length"], np.float32),
                        l0=np.asarray(cells["l0"], np.float32), diameter=np.asarray(cells["diameter"], np.float32),
                        age=np.asarray(cells["age"], np.int32), dt=np.float64(dt), steps=np.int64(steps),
                        seed=np.int64(seed), radius=np.float64(last.get("colony_radius", 0.0)),
                        tail_bbpgd=np.array([t["bbpgd_iterations"] for t in tail], np.int64),
                        tail_relcp=np.array([t["relcp_iterations"] for t in tail], np.int64),
                        tail_cells=np.array([t["n_cells"] for t in tail], np.int64))


def load_snapshot(path: str) -> tuple[dict, float, dict]:
    """Cells of a saved grown colony (float64, planar: z = 0, rotation about z)
    and the time step it ended with."""
    d = np.load(path)
    th = d["theta"].astype(np.float64)
    n = th.size
    cells = {"x": d["x"].astype(np.float64), "y": d["y"].astype(np.float64), "z": np.zeros(n),
             "q0": np.cos(th / 2), "q1": np.zeros(n), "q2": np.zeros(n), "q3": np.sin(th / 2),
             "length": d["length"].astype(np.float64), "l0": d["l0"].astype(np.float64),
             "diameter": d["diameter"].astype(np.float64), "age": d["age"].astype(np.int32)}
    meta = {k: d[k].tolist() for k in d.files if k not in cells and k != "theta"}
    return cells, float(d["dt"]), meta


def colony_jobs(n: int, rng, r_min: float, r_max: float, hard_frac: float, arrivals=None) -> list[dict]:
    """Colony jobs as in the batch sweep / serving configs: sequential seeds,
    growth rate g ~ U[0.5, 1.5] (tau = 1/g), R_end log-uniform in [r_min, r_max],
    hard jobs with CFL-adaptive dt capped at 1e-3, soft jobs at dt = 3e-5 with
    the Hertz constant of E = 1e3, R_eff = 0.125."""
    jobs = []
    for k in range(n):
        hard = rng.random() < hard_frac
        g = rng.uniform(0.5, 1.5)
        r_end = float(np.exp(rng.uniform(np.log(r_min), np.log(r_max))))
        if hard:
            p = abi.default_params(mode=abi.MODE_HARD, seed=k, tau=1.0 / g, dt=1e-3, fixed_dt=0, dt_cap=1e-3)
        else:
            p = abi.default_params(mode=abi.MODE_SOFT, seed=k, tau=1.0 / g, dt=3e-5, fixed_dt=1,
                                   kcc=1333.3333333333333)
        jobs.append({"params": p, "end_radius": r_end, "arrival_s": 0.0 if arrivals is None else arrivals[k],
                     "hard": hard})
    return jobs


def run_jobs(args):
    """Batch sweep (--jobs N, all arrive at once) or serving (--rate R jobs/s,
    Poisson arrivals for --serve-seconds): continuous batching with --slots
    colonies in flight, against a sample of the same jobs one at a time."""
    from pcc_b200 import build, device
    build.build()
    rng = np.random.default_rng(args.job_seed)
    if args.rate > 0:
        t, arr = 0.0, []
        while True:
            t += rng.exponential(1.0 / args.rate)
            if t > args.serve_seconds:
                break
            arr.append(t)
        jobs = colony_jobs(len(arr), rng, args.r_min, args.r_max, args.hard_frac, arr)
    else:
        jobs = colony_jobs(args.jobs, rng, args.r_min, args.r_max, args.hard_frac)
    prec = abi.PRECISION_MIXED if args.precision == "mixed" else abi.PRECISION_FP64
    for j in jobs:
        j["params"].max_bbpgd_iterations = args.max_bbpgd
        if j["hard"]:
            j["params"].precision = prec
    res, wall = device.serve(jobs, slots=args.slots, hbm_budget_bytes=args.hbm_budget, check=False)
    failed = [dict(job=k, status=abi.STATUS_NAMES.get(r["status"], r["status"]), steps=r["steps"], cells=r["cells"],
                   radius=r["radius"], dt=r["dt"], r_end=jobs[k]["end_radius"], hard=jobs[k]["hard"],
                   tau=jobs[k]["params"].tau, max_step_bbpgd=r["max_step_bbpgd"])
              for k, r in enumerate(res) if r["status"] != 0]
    lat = np.array([r["finish_s"] - r["arrival_s"] for r in res])
    cells = sum(r["cell_steps"] for r in res)
    # baseline: a size-stratified sample of the same jobs (evenly spaced in
    # R_end order) one at a time on the plain FP64 path
    order = sorted(range(len(jobs)), key=lambda k: jobs[k]["end_radius"])
    nb = min(args.baseline_jobs, len(jobs))
    picked = sorted({order[int(round(i * (len(order) - 1) / max(nb - 1, 1)))] for i in range(nb)})
    sample = []
    for k in picked:
        q = abi.Params.from_buffer_copy(jobs[k]["params"])
        q.precision = abi.PRECISION_FP64
        sample.append(dict(jobs[k], params=q, arrival_s=0.0))
    res1, wall1 = device.serve(sample, slots=1, hbm_budget_bytes=args.hbm_budget, check=False)
    seq_rate = sum(r["cell_steps"] for r in res1) / wall1
    # every sampled job alone with the mix's own settings: results must be identical
    if prec == abi.PRECISION_FP64:
        alone = res1
    else:
        alone, _ = device.serve([dict(jobs[k], arrival_s=0.0) for k in picked], slots=1,
                                hbm_budget_bytes=args.hbm_budget, check=False)
    same = all(a["checksum"] == res[k]["checksum"] and a["steps"] == res[k]["steps"] and
               a["status"] == res[k]["status"] for a, k in zip(alone, picked))
    line = {
        "metric": METRIC, "mode": "serve" if args.rate > 0 else "batch",
        "jobs": len(jobs), "hard_jobs": sum(j["hard"] for j in jobs), "slots": args.slots,
        "offered_jobs_per_s": args.rate if args.rate > 0 else None,
        "colonies_per_s": len(jobs) / wall, "cell_steps_per_s": cells / wall, "wall_s": wall,
        "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                      "max": float(lat.max())},
        "one_at_a_time": {"jobs": len(sample), "cell_steps_per_s": seq_rate, "wall_s": wall1,
                          "r_end": [jobs[k]["end_radius"] for k in picked],
                          "path": "plain FP64, one job at a time (slots = 1), sample evenly spaced in R_end"},
        "identity_checked_jobs": len(picked),
        "speedup_vs_one_at_a_time": (cells / wall) / seq_rate,
        "results_identical_alone_and_in_mix": same,
        "max_step_bbpgd": int(max(r["max_step_bbpgd"] for r in res)),
        "failed_jobs": failed,
        "config": {"r_end": [args.r_min, args.r_max], "growth_rate": [0.5, 1.5], "hard_fraction": args.hard_frac,
                   "hbm_budget_bytes": args.hbm_budget, "tolerance": 1e-3,
                   "dtype": "f64" if prec == abi.PRECISION_FP64 else "hard jobs mixed (f32 operands, f64 accumulation)"},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--radius", type=float, default=RADIUS)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-small", action="store_true", help="skip the config 0 / config 1 runs")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed",
                    help="BBPGD operand precision (mixed: FP32 D/L/M/U, FP64 gamma, dots, residual)")
    ap.add_argument("--verbose", action="store_true", help="per-step solver statistics on stderr")
    ap.add_argument("--frozen", action="store_true", help="BBPGD microbench on a frozen constraint set")
    ap.add_argument("--frozen-tol", type=float, default=1e-3, help="--frozen: BBPGD tolerance of the frozen solves")
    ap.add_argument("--start", choices=["packing", "grown"], default="packing",
                    help="--frozen: the synthetic dense packing of --radius, or the grown R=260 colony")
    ap.add_argument("--jobs", type=int, default=0, help="batch sweep of N colonies (continuous batching)")
    ap.add_argument("--rate", type=float, default=0.0, help="serving: Poisson arrivals per second")
    ap.add_argument("--serve-seconds", type=float, default=10.0)
    ap.add_argument("--slots", type=int, default=32)
    ap.add_argument("--r-min", type=float, default=10.0)
    ap.add_argument("--r-max", type=float, default=20.0)
    ap.add_argument("--hard-frac", type=float, default=0.8)
    ap.add_argument("--hbm-budget", type=float, default=150e9)
    ap.add_argument("--baseline-jobs", type=int, default=8)
    ap.add_argument("--job-seed", type=int, default=0)
    ap.add_argument("--max-bbpgd", type=int, default=500000, help="BBPGD iteration cap of each job")
    ap.add_argument("--grow", action="store_true", help="grow one colony from a single cell to --radius")
    ap.add_argument("--grow-seconds", type=float, default=1500.0, help="wall-clock limit of --grow")
    ap.add_argument("--save", default="", help="--grow: save the final colony (npz) as a benchmark start state")
    ap.add_argument("--checkpoint", default="", help="--grow: save the exact final state and run totals (npz)")
    ap.add_argument("--resume", default="", help="--grow: continue the run saved by --checkpoint")
    ap.add_argument("--replica-selftest", action="store_true", help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(spawn_ranks(args.gpus))
    if args.replica_selftest:
        run_replica_selftest(args)
    elif args.grow:
        run_grow(args)
    elif args.jobs > 0 or args.rate > 0:
        run_jobs(args)
    elif args.frozen:
        run_frozen(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
