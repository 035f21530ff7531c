"""Benchmark of the collision hot path: cell-steps/s of the hard model.

Workload (default): one colony of radius 260 in the hard model, FP64, the
scale of the reference's largest published run (R = 260).  The colony is a
synthetic, deterministic dense packing (pcc_b200.synth.dense_colony: ~2.2e5
rod cells in orientation domains, every neighbour touching), since growing a
real one takes hours; a step is one full simulator step on it through the C
ABI -- divide, x-sort renumbering, the ReLCP loop of contact detection and
BBPGD solves, motion, growth and the CFL time-step adaptation (dt starts at
3e-4, capped at 1e-3).  value = sum of cells over the K timed steps / device
time (CUDA events on the library's stream), summed over ranks; each rank runs
its own colony (replicas, no collective on the data path: weak scaling).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference simulator's own C++ code (compiled in
place against single-rank PETSc/MPI stand-ins, oracle/_ref/libpccref_fast.so,
release flags) on a bounded sample of the same workload on the host cores.
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
CPU_SAMPLE_RADIUS = 40.0  # bounded sample for the CPU legs (~5e3 cells)
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


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def reduce_max(world: int, v: float) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(world: int, v: float) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def aggregate(cells_per_rank: list[float], ms_per_rank: list[float]) -> tuple[float, float]:
    """Whole-job throughput: all ranks' cell-steps over the slowest rank's time."""
    t = max(ms_per_rank)
    return sum(cells_per_rank) / (t / 1e3), t


def cpu_rate(fast_ref: bool, seconds: float = 15.0, radius: float = CPU_SAMPLE_RADIUS, min_steps: int = 2,
             max_steps: int | None = None, warmup: int = 1):
    """cell-steps/s of a CPU implementation on a bounded sample of the workload."""
    sys.path.insert(0, str(ROOT / "tests"))
    from oracles import OracleColony, RefColony
    kind = "port"
    p = colony_params()
    col = None
    if fast_ref and (ROOT / "oracle" / "_ref" / "libpccref_fast.so").exists():
        col = RefColony(p, fast=True)
        kind = "reference"
    else:
        col = OracleColony(p)
    cells = make_colony(radius, seed=0)
    col.set_cells(cells)
    for _ in range(warmup):
        col.step()
    t0 = time.perf_counter()
    cs, k = 0.0, 0
    while (time.perf_counter() - t0 < seconds or k < min_steps) and (max_steps is None or k < max_steps):
        cs += col.step()["n_cells"]
        k += 1
    el = time.perf_counter() - t0
    return cs / el, kind, k, len(cells["x"]), el


def run_reference(args):
    world, rank, _ = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0
    if rank != 0:
        return
    rate, kind, k, n, el = cpu_rate(True, seconds=1e9, min_steps=args.steps, max_steps=args.steps,
                                    warmup=args.warmup)
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / k * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "hard model colony step, FP64 (bounded sample)", "radius": CPU_SAMPLE_RADIUS,
                   "cells": n, "parallelism": "1 rank, 1 thread"},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": 1, "kind": kind,
                         "sample": f"{k} steps of the synthetic dense colony at R={CPU_SAMPLE_RADIUS:g} "
                                   f"({n} cells) after {args.warmup} warm-up steps"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    world, rank, local = dist_setup()
    from pcc_b200 import build, device
    if rank == 0:
        build.build()
    barrier(world)
    import torch
    torch.cuda.init()
    cells = make_colony(args.radius, seed=rank)
    prec = abi.PRECISION_MIXED if args.precision == "mixed" else abi.PRECISION_FP64
    p = colony_params(capacity_hint=int(len(cells["x"]) * 1.5), precision=prec)
    col = device.Colony(p, device=local)
    col.set_cells(cells)
    stream = torch.cuda.ExternalStream(col.stream, device=f"cuda:{local}")
    for _ in range(args.warmup):
        col.step()
    errors = precision_errors(device, col, p, local) if rank == 0 and prec == abi.PRECISION_MIXED else None
    col.profiling(True)
    launches0 = col.launches
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    hist = []
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            hist.append(col.step())
            if args.verbose:
                print(json.dumps(hist[-1]), file=sys.stderr, flush=True)
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    ms = e0.elapsed_time(e1)
    launches = col.launches - launches0
    prof = col.profile()
    cells_steps = float(sum(h["n_cells"] for h in hist))
    ms_max = reduce_max(world, ms)
    total = reduce_sum(world, cells_steps)
    value = total / (ms_max / 1e3)

    # end to end through the C ABI with host buffers: upload the state from
    # pinned host memory, step, read the state back, every step
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
    e2e_total = reduce_sum(world, e2e_cells)
    e2e_value = e2e_total / (e2e_ms / 1e3)

    peaks = measured_peaks()
    bb_ms = prof["bbpgd_ms"]
    achieved = prof["bbpgd_algo_bytes"] / (bb_ms / 1e3) / 1e9 if bb_ms > 0 else 0.0
    mixed = prec == abi.PRECISION_MIXED
    ratio = traffic_ratio("k_bbpgd_planar_mixed_frozen_r260" if mixed else "k_bbpgd_planar_frozen_r260")
    launches_bb = max(prof["bbpgd_launches"], 1)
    traffic = ratio * prof["bbpgd_algo_bytes"] / launches_bb if ratio else None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if prec == abi.PRECISION_FP64 else "f32 operands / f64 accumulation",
        "data": "synthetic",
        "config": {"workload": f"hard model colony step, {'FP64' if prec == abi.PRECISION_FP64 else 'mixed precision'}"
                               f", synthetic dense colony R={args.radius:g}",
                   "cells_per_rank": int(hist[0]["n_cells"]), "ghost_mode": "single_rank",
                   "tolerance": p.tolerance, "dt_start": 3e-4, "dt_cap": 1e-3,
                   "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (state + constraints > 126 MB per step)"},
        "roofline": {"bound": "hbm", "achieved": achieved,
                     "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"] if peaks.get("hbm_gbs") else None,
                     "traffic": traffic,
                     "kernel": f"k_bbpgd_planar<{'float' if mixed else 'double'}> (persistent BBPGD)",
                     "peak_source": "fallback" if peaks.get("fallback") else "measured"},
        "bbpgd_iterations_per_s": prof["bbpgd_iterations"] / (ms / 1e3),
        "bbpgd_iterations_per_step": prof["bbpgd_iterations"] / max(args.steps, 1),
        "stage_ms": {"bbpgd": bb_ms, "detect": prof["detect_ms"], "solve": prof["solve_ms"], "total": ms},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d // e2e_steps,
                "d2h_bytes_per_step": d2h // e2e_steps},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    if errors is not None:
        line["mixed_vs_fp64"] = errors
    if rank == 0 and world == 1 and not args.no_cpu:
        # one step of the same colony (~20 s of CPU work at R = 260): the first
        # step from the packing, FP64, the reference's own code at release flags
        rate, kind, k, ncpu, el = cpu_rate(True, seconds=0.0, radius=args.radius, min_steps=1, max_steps=1,
                                           warmup=0)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": 1, "kind": kind,
                                "sample": f"{k} step ({el:.1f} s) of the same synthetic dense colony at "
                                          f"R={args.radius:g} ({ncpu} cells), the first step from the packing, "
                                          f"FP64; one rank, one thread (the reference has no threaded path "
                                          f"and no MPI is available)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    col.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


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
    cells = make_colony(args.radius, seed=0)
    prec = abi.PRECISION_MIXED if args.precision == "mixed" else abi.PRECISION_FP64
    col = device.Colony(colony_params(capacity_hint=int(len(cells["x"]) * 1.5), precision=prec))
    col.set_cells(cells)
    for _ in range(args.warmup):
        col.step()
    n = col.n_cells
    col.profiling(True)
    it, res, ms = col.bbpgd_frozen(3e-4, max(args.steps, 1))
    prof = col.profile()
    bc, bn = ALGO_BYTES[args.precision]
    m = int(round((prof["bbpgd_algo_bytes"] / max(prof["bbpgd_iterations"], 1) - bn * n) / bc))
    algo = it * (bc * m + bn * n)
    print(json.dumps({"frozen_bbpgd": True, "precision": args.precision, "radius": args.radius, "cells": n, "constraints": m, "iterations": it,
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
    p = colony_params(dt=1e-3, precision=prec, capacity_hint=int(4.5 * args.radius ** 2 * 1.2) + 64)
    col = device.Colony(p)
    col.set_cells(abi.seed_cell(args.job_seed))
    stream = torch.cuda.ExternalStream(col.stream, device="cuda:0")
    col.profiling(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.time()
    tlast = t0
    steps = bb = 0
    cells = 0.0
    radius = 0.0
    marks = []
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
            marks.append({"radius": radius, "step": steps, "cells": st["n_cells"], "wall_s": time.time() - t0,
                          "dt": st["dt_used"], "bbpgd_step": st["bbpgd_iterations"]})
        if time.time() - tlast > 10:
            tlast = time.time()
            print(json.dumps({"step": steps, "radius": radius, "cells": st["n_cells"], "dt": st["dt_used"],
                              "bbpgd": st["bbpgd_iterations"], "wall_s": tlast - t0}), file=sys.stderr, flush=True)
        tail.append(st)
    e1.record(stream)
    e1.synchronize()
    wall = time.time() - t0
    dev_ms = e0.elapsed_time(e1)
    prof = col.profile()
    final = col.get_cells()
    if args.save:
        save_snapshot(args.save, final, col.dt, steps, st, tail, args.job_seed)
    print(json.dumps({
        "grow": True, "precision": args.precision, "radius_target": args.radius, "radius": radius,
        "reached": radius >= args.radius, "steps": steps, "cells": int(st.get("n_cells", 1)),
        "cell_steps": cells, "wall_s": wall, "device_s": dev_ms / 1e3, "cell_steps_per_s": cells / (dev_ms / 1e3),
        "bbpgd_iterations": bb, "bbpgd_iterations_per_s": bb / (dev_ms / 1e3),
        "stage_ms": {"bbpgd": prof["bbpgd_ms"], "detect": prof["detect_ms"], "solve": prof["solve_ms"]},
        "packing_fraction": packing_fraction(final), "sim_time": st.get("sim_time"), "marks": marks,
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
    # baseline: a sample of the same jobs one at a time on the plain FP64 path
    sample = []
    for j in jobs[: args.baseline_jobs]:
        q = abi.Params.from_buffer_copy(j["params"])
        q.precision = abi.PRECISION_FP64
        sample.append(dict(j, params=q, arrival_s=0.0))
    res1, wall1 = device.serve(sample, slots=1, hbm_budget_bytes=args.hbm_budget, check=False)
    seq_rate = sum(r["cell_steps"] for r in res1) / wall1
    # the same jobs alone with the mix's own settings: results must be identical
    if prec == abi.PRECISION_FP64:
        alone = res1
    else:
        alone, _ = device.serve([dict(j, arrival_s=0.0) for j in jobs[: min(2, args.baseline_jobs)]], slots=1,
                                hbm_budget_bytes=args.hbm_budget, check=False)
    same = all(a["checksum"] == b["checksum"] and a["steps"] == b["steps"] and a["status"] == b["status"]
               for a, b in zip(alone, res))
    line = {
        "metric": METRIC, "mode": "serve" if args.rate > 0 else "batch",
        "jobs": len(jobs), "hard_jobs": sum(j["hard"] for j in jobs), "slots": args.slots,
        "offered_jobs_per_s": args.rate if args.rate > 0 else None,
        "colonies_per_s": len(jobs) / wall, "cell_steps_per_s": cells / wall, "wall_s": wall,
        "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                      "max": float(lat.max())},
        "one_at_a_time": {"jobs": len(sample), "cell_steps_per_s": seq_rate, "wall_s": wall1,
                          "path": "plain FP64, one job at a time (slots = 1)"},
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
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--radius", type=float, default=RADIUS)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed",
                    help="BBPGD operand precision (mixed: FP32 D/L/M/U, FP64 gamma, dots, residual)")
    ap.add_argument("--verbose", action="store_true", help="per-step solver statistics on stderr")
    ap.add_argument("--frozen", action="store_true", help="BBPGD microbench on a frozen constraint set")
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
    args = ap.parse_args()
    if args.grow:
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
