"""Generates the golden fixtures in this folder from the reference simulator
itself: its own C++ sources compiled in place against single-rank PETSc/MPI
stand-ins (oracle/_ref/libpccref_strict.so, built by `make -C oracle ref`
while the reference tree is mounted).

Run from the repository root:  python tests/golden/make_golden.py [name ...]
(no names: every fixture).
Each fixture is a compressed .npz holding the inputs (a colony snapshot and
parameters) and the reference's outputs on them.  The GPU box has no copy of
the reference; the tests there read these files.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))
import pcc_pkg  # noqa: E402

pcc_pkg.load_package()
from pcc_b200 import abi  # noqa: E402
from oracles import RefColony, ref_division_length  # noqa: E402

OUT = Path(__file__).resolve().parent
PARAM_KEYS = [k for k, _ in abi.Params._fields_]


def params_dict(p: abi.Params) -> dict:
    return {k: getattr(p, k) for k in PARAM_KEYS}


def pack(prefix: str, d: dict, out: dict):
    for k, v in d.items():
        out[f"{prefix}{k}"] = np.asarray(v)


def grow(p: abi.Params, seed: int, radius: float, max_steps: int = 10**7):
    r = RefColony(p)
    r.set_cells(abi.seed_cell(seed))
    stats = []
    while r.colony_radius < radius and len(stats) < max_steps:
        stats.append(r.step())
    return r, stats


def snapshot_fixture(name: str, mode: int, seed: int, radius: float, dt: float, kcc: float, ghost: int):
    p = abi.default_params(dt=dt, fixed_dt=1, seed=seed, mode=mode, ghost_mode=ghost, kcc=kcc)
    r, stats = grow(p, seed, radius)
    out: dict = {}
    snap = r.get_cells()
    pack("cells_", snap, out)
    out["params"] = np.array([params_dict(p)], dtype=object)
    out["division_count"] = np.array(r.division_count)
    # contact lists on the snapshot (phase-0 and later-phase tolerances, soft 0)
    for tag, tol in (("det25_", 0.25), ("dettol_", p.tolerance), ("det0_", 0.0)):
        pack(tag, r.detect(tol, 0), out)
    # one solver call on the snapshot
    r2 = RefColony(p)
    r2.set_cells(snap)
    st = r2.solve(dt, 0)
    out["solve_stats"] = np.array([st], dtype=object)
    pack("solve_cells_", r2.get_cells(), out)
    pack("solve_cons_", r2.constraints(), out)
    # growth history up to the snapshot
    out["hist_n_cells"] = np.array([s["n_cells"] for s in stats])
    out["hist_bbpgd"] = np.array([s["bbpgd_iterations"] for s in stats])
    out["hist_relcp"] = np.array([s["relcp_iterations"] for s in stats])
    out["hist_ncons"] = np.array([s["n_constraints"] for s in stats])
    np.savez_compressed(OUT / f"{name}.npz", **out)
    print(name, len(snap["x"]), "cells", len(stats), "steps", out["det25_sd"].size, "contacts")


def solve_fixture(name: str, p: abi.Params, snap: dict, dt: float):
    """One solver call of the mode in `p` on a given snapshot."""
    out: dict = {}
    pack("cells_", snap, out)
    out["params"] = np.array([params_dict(p)], dtype=object)
    r = RefColony(p)
    r.set_cells(snap)
    pack("det0_", r.detect(0.0, 0), out)
    r.set_cells(snap)
    st = r.solve(dt, 0)
    out["solve_stats"] = np.array([st], dtype=object)
    pack("solve_cells_", r.get_cells(), out)
    pack("solve_cons_", r.constraints(), out)
    np.savez_compressed(OUT / f"{name}.npz", **out)
    print(name, len(snap["x"]), "cells", out["det0_sd"].size, "contacts")


def trajectory_fixture(name: str, mode: int, seed: int, steps: int, dt: float, kcc: float, ghost: int, fixed: int,
                       start: dict | None = None):
    p = abi.default_params(dt=dt, fixed_dt=fixed, seed=seed, mode=mode, ghost_mode=ghost, kcc=kcc)
    r = RefColony(p)
    cells0 = start if start is not None else abi.seed_cell(seed)
    r.set_cells(cells0)
    stats = [r.step() for _ in range(steps)]
    out: dict = {}
    pack("start_", cells0, out)
    pack("final_", r.get_cells(), out)
    out["params"] = np.array([params_dict(p)], dtype=object)
    for k in ("n_cells", "bbpgd_iterations", "relcp_iterations", "n_constraints", "residual", "max_overlap",
              "dt_used", "colony_radius", "n_divided"):
        out[f"hist_{k}"] = np.array([s[k] for s in stats])
    np.savez_compressed(OUT / f"{name}.npz", **out)
    print(name, steps, "steps ->", stats[-1]["n_cells"], "cells")


HIST_KEYS = ("n_cells", "bbpgd_iterations", "relcp_iterations", "n_constraints", "residual", "max_overlap",
             "dt_used", "colony_radius", "n_divided")
LIGHT_CONS = ("gid_i", "gid_j", "sd", "gamma", "phase")


def one_solve(p: abi.Params, snap: dict, dt: float, out: dict, prefix: str, light: bool = False):
    """The reference's solver call on `snap` (fresh handle: division stream and
    Brownian generator at their start) stored under `prefix`; `light` keeps
    only the ids, phi, gamma and phase of the returned constraints."""
    r = RefColony(p)
    r.set_cells(snap)
    st = r.solve(dt, 0)
    out[f"{prefix}stats"] = np.array([st], dtype=object)
    pack(f"{prefix}cells_", r.get_cells(), out)
    cons = r.constraints()
    if light:
        cons = {k: cons[k] for k in LIGHT_CONS}
    pack(f"{prefix}cons_", cons, out)


def continuation(p: abi.Params, snap: dict, dt: float, steps: int, out: dict, prefix: str):
    """`steps` full steps from `snap` on a fresh reference handle."""
    r = RefColony(p)
    r.set_cells(snap)
    r.dt = dt
    stats = [r.step() for _ in range(steps)]
    pack(f"{prefix}final_", r.get_cells(), out)
    for k in HIST_KEYS:
        out[f"{prefix}hist_{k}"] = np.array([s[k] for s in stats])


def grown_fixture(name: str, p: abi.Params, radius: float, mid_cells: int, cont_steps: int):
    """A colony grown by the reference from one cell (orientation from p.seed)
    to `radius`, with its per-step history; the first state past `mid_cells`
    and the final state as snapshots, each with the reference's contact lists,
    one solver call and a short continuation from it."""
    r = RefColony(p)
    r.set_cells(abi.seed_cell(int(p.seed)))
    stats, mid, mid_dt = [], None, None
    while r.colony_radius < radius:
        stats.append(r.step())
        if mid is None and stats[-1]["n_cells"] >= mid_cells:
            mid, mid_dt = r.get_cells(), r.dt
    end, end_dt = r.get_cells(), r.dt
    out: dict = {"params": np.array([params_dict(p)], dtype=object)}
    for k in HIST_KEYS:
        out[f"hist_{k}"] = np.array([s[k] for s in stats])
    for tag, snap, dt in (("mid_", mid, mid_dt), ("end_", end, end_dt)):
        pack(f"{tag}cells_", snap, out)
        out[f"{tag}dt"] = np.array(dt)
        r2 = RefColony(p)
        r2.set_cells(snap)
        for dtag, tol in (("det25_", 0.25), ("dettol_", p.tolerance), ("det0_", 0.0)):
            pack(f"{tag}{dtag}", r2.detect(tol, 0), out)
        one_solve(p, snap, dt, out, f"{tag}solve_")
        continuation(p, snap, dt, cont_steps, out, f"{tag}cont_")
    np.savez_compressed(OUT / f"{name}.npz", **out)
    print(name, len(stats), "steps;", len(mid["x"]), "and", len(end["x"]), "cells")


def dense_fixture(name: str, radius: float, seed: int, cont_steps: int, lists=("det25_", "dettol_", "det0_")):
    """The benchmark's synthetic dense colony (synth.dense_colony, neighbours
    touching) at `radius`: contact lists, one hard solve with the benchmark's
    parameters, one soft solve with the Hertz constant of E = 1e3, R_eff = 0.125,
    and a few hard steps with CFL-adaptive dt."""
    from pcc_b200 import synth
    cells = synth.dense_colony(radius, seed=seed, lane_gap=0.0, end_gap=0.0)
    hard = abi.default_params(dt=3e-4, fixed_dt=0, dt_cap=1e-3, mode=abi.MODE_HARD, ghost_mode=abi.GHOSTS_SINGLE_RANK,
                              seed=seed)
    soft = abi.default_params(dt=3e-5, fixed_dt=1, mode=abi.MODE_SOFT, ghost_mode=abi.GHOSTS_SINGLE_RANK, seed=seed,
                              kcc=1333.3333333333333)
    out: dict = {"params": np.array([params_dict(hard)], dtype=object),
                 "soft_params": np.array([params_dict(soft)], dtype=object)}
    pack("cells_", cells, out)
    r = RefColony(hard)
    r.set_cells(cells)
    for dtag, tol in (("det25_", 0.25), ("dettol_", hard.tolerance), ("det0_", 0.0)):
        if dtag in lists:
            pack(dtag, r.detect(tol, 0), out)
    one_solve(hard, cells, hard.dt, out, "solve_", light=True)
    one_solve(soft, cells, soft.dt, out, "soft_solve_", light=True)
    continuation(hard, cells, hard.dt, cont_steps, out, "cont_")
    np.savez_compressed(OUT / f"{name}.npz", **out)
    print(name, len(cells["x"]), "cells", out["det25_sd"].size, "phase-0 contacts")


def tight_fixture(name: str, source: str, prefix: str, tolerance: float):
    """One reference solver call at a tight tolerance on a snapshot of another
    fixture: both solvers then converge to the same LCP solution, which pins
    the device's solve beyond the 1e-3 tolerance at which two valid solutions
    may differ by about the tolerance."""
    src = np.load(OUT / f"{source}.npz", allow_pickle=True)
    snap = {k[len(f"{prefix}cells_"):]: src[k] for k in src.files if k.startswith(f"{prefix}cells_")}
    p = abi.default_params()
    for k, v in src["params"][0].items():
        setattr(p, k, v)
    p.tolerance = tolerance
    dt = float(src[f"{prefix}dt"])
    out: dict = {"params": np.array([params_dict(p)], dtype=object), "dt": np.array(dt)}
    pack("cells_", snap, out)
    one_solve(p, snap, dt, out, "solve_", light=True)
    np.savez_compressed(OUT / f"{name}.npz", **out)
    print(name, len(snap["x"]), "cells", out["solve_stats"][0])


def soft_grown_fixture(name: str, p: abi.Params, radius: float):
    """A soft-model colony grown by the reference from one cell to `radius`
    (the cell-count history of every step, the radius every 1000 steps, the
    final state and one force assembly on it)."""
    r = RefColony(p)
    r.set_cells(abi.seed_cell(int(p.seed)))
    n_cells, radii = [], []
    while r.colony_radius < radius:
        st = r.step()
        n_cells.append(st["n_cells"])
        if len(n_cells) % 1000 == 0:
            radii.append(st["colony_radius"])
    out: dict = {"params": np.array([params_dict(p)], dtype=object), "hist_n_cells": np.array(n_cells, np.int32),
                 "hist_radius_every_1000": np.array(radii)}
    end = r.get_cells()
    pack("end_cells_", end, out)
    one_solve(p, end, p.dt, out, "end_solve_", light=True)
    np.savez_compressed(OUT / f"{name}.npz", **out)
    print(name, len(n_cells), "steps ->", len(end["x"]), "cells")


def brownian_fixture(name: str):
    """Brownian kicks (temperature > 0): two solver calls in a row on the
    R = 10 snapshot (the generator stream continues), hard and soft, monolayer
    and out-of-plane, and a growth trajectory from one cell."""
    hard = np.load(OUT / "hard_r10_seed3.npz", allow_pickle=True)
    snap = {k[len("cells_"):]: hard[k] for k in hard.files if k.startswith("cells_")}
    out: dict = {}
    pack("cells_", snap, out)
    cases = {
        "hard_": abi.default_params(dt=1e-3, fixed_dt=1, seed=3, temperature=0.5),
        "hard3d_": abi.default_params(dt=1e-3, fixed_dt=1, seed=3, temperature=0.5, monolayer=0),
        "soft_": abi.default_params(dt=3e-5, fixed_dt=1, seed=3, temperature=0.5, mode=abi.MODE_SOFT,
                                    kcc=1333.3333333333333),
    }
    for tag, p in cases.items():
        out[f"{tag}params"] = np.array([params_dict(p)], dtype=object)
        r = RefColony(p)
        r.set_cells(snap)
        for k in (1, 2):
            st = r.solve(p.dt, 0)
            out[f"{tag}solve{k}_stats"] = np.array([st], dtype=object)
            pack(f"{tag}solve{k}_cells_", r.get_cells(), out)
    p = abi.default_params(dt=1e-3, fixed_dt=1, seed=7, temperature=0.2)
    out["traj_params"] = np.array([params_dict(p)], dtype=object)
    r = RefColony(p)
    r.set_cells(abi.seed_cell(7))
    stats = [r.step() for _ in range(1500)]
    pack("traj_final_", r.get_cells(), out)
    for k in HIST_KEYS:
        out[f"traj_hist_{k}"] = np.array([s[k] for s in stats])
    np.savez_compressed(OUT / f"{name}.npz", **out)
    print(name, "final trajectory cells", stats[-1]["n_cells"])


def division_fixture():
    seeds, ks, lens, vals = [], [], [], []
    for seed in (0, 1, 3, 12345, 2**63 + 7):
        for k in range(6):
            for L in (2.0, 1.999999999, 2.0000001, 1.5, 3.25):
                seeds.append(seed)
                ks.append(k)
                lens.append(L)
                vals.append(ref_division_length(seed, k, L))
    np.savez_compressed(OUT / "division_draws.npz", seed=np.array(seeds, dtype=np.uint64), k=np.array(ks),
                        length=np.array(lens), value=np.array(vals))
    print("division_draws", len(vals))


FIXTURES = {
    "division_draws": division_fixture,
    "hard_r10_seed3": lambda: snapshot_fixture("hard_r10_seed3", abi.MODE_HARD, 3, 10.0, 1e-3, 20000.0,
                                               abi.GHOSTS_SINGLE_RANK),
    "hard_r5_seed0_noghost": lambda: snapshot_fixture("hard_r5_seed0_noghost", abi.MODE_HARD, 0, 5.0, 1e-3, 20000.0,
                                                      abi.GHOSTS_NONE),
    "soft_on_hard_r10_seed3": lambda: solve_fixture(
        "soft_on_hard_r10_seed3", abi.default_params(dt=3e-5, fixed_dt=1, seed=3, mode=abi.MODE_SOFT,
                                                     ghost_mode=abi.GHOSTS_SINGLE_RANK, kcc=1333.3333333333333),
        _r10_snapshot(), 3e-5),
    "hard_tight_r10_seed3": lambda: solve_fixture(
        "hard_tight_r10_seed3", abi.default_params(dt=1e-3, fixed_dt=1, seed=3, mode=abi.MODE_HARD,
                                                   ghost_mode=abi.GHOSTS_SINGLE_RANK, tolerance=1e-6),
        _r10_snapshot(), 1e-3),
    "soft_r3_seed1": lambda: snapshot_fixture("soft_r3_seed1", abi.MODE_SOFT, 1, 3.0, 3e-5, 1333.3333333333333,
                                              abi.GHOSTS_SINGLE_RANK),
    "traj_hard_seed3_3000": lambda: trajectory_fixture("traj_hard_seed3_3000", abi.MODE_HARD, 3, 3000, 1e-3, 20000.0,
                                                       abi.GHOSTS_SINGLE_RANK, 1),
    "traj_hard_adaptive_seed5_2000": lambda: trajectory_fixture("traj_hard_adaptive_seed5_2000", abi.MODE_HARD, 5,
                                                                2000, 1e-2, 20000.0, abi.GHOSTS_SINGLE_RANK, 0),
    # hard, FP64, dt = 1e-3 fixed, grown from one cell to R = 20 (~1.6e3 cells)
    "grown_hard_r20_seed0": lambda: grown_fixture(
        "grown_hard_r20_seed0", abi.default_params(dt=1e-3, fixed_dt=1, seed=0, mode=abi.MODE_HARD,
                                                   ghost_mode=abi.GHOSTS_SINGLE_RANK), 20.0, 1100, 10),
    "dense_r20_seed0": lambda: dense_fixture("dense_r20_seed0", 20.0, 0, 5),
    "dense_r40_seed0": lambda: dense_fixture("dense_r40_seed0", 40.0, 0, 3, lists=("det25_",)),
    # soft, dt = 3e-5, E = 1e3 and R_eff = 0.125 (kcc = 4/3 E), grown from one cell to R = 20
    "grown_soft_r20_seed0": lambda: soft_grown_fixture(
        "grown_soft_r20_seed0", abi.default_params(dt=3e-5, fixed_dt=1, seed=0, mode=abi.MODE_SOFT,
                                                   ghost_mode=abi.GHOSTS_SINGLE_RANK, kcc=1333.3333333333333), 20.0),
    "brownian_r10_seed3": lambda: brownian_fixture("brownian_r10_seed3"),
    # the 1,100-cell snapshot of grown_hard_r20_seed0 solved at tolerance 1e-6
    "grown_hard_r20_tight": lambda: tight_fixture("grown_hard_r20_tight", "grown_hard_r20_seed0", "mid_", 1e-6),
}


def _r10_snapshot() -> dict:
    hard = np.load(OUT / "hard_r10_seed3.npz", allow_pickle=True)
    return {k[len("cells_"):]: hard[k] for k in hard.files if k.startswith("cells_")}


def main(names: list[str]):
    for name in names or list(FIXTURES):
        FIXTURES[name]()


if __name__ == "__main__":
    main(sys.argv[1:])
