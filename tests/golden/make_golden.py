"""Generates the golden fixtures in this folder from the reference simulator
itself: its own C++ sources compiled in place against single-rank PETSc/MPI
stand-ins (oracle/_ref/libpccref_strict.so, built by `make -C oracle ref`
while the reference tree is mounted).

Run from the repository root:  python tests/golden/make_golden.py
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


def main():
    division_fixture()
    snapshot_fixture("hard_r10_seed3", abi.MODE_HARD, 3, 10.0, 1e-3, 20000.0, abi.GHOSTS_SINGLE_RANK)
    snapshot_fixture("hard_r5_seed0_noghost", abi.MODE_HARD, 0, 5.0, 1e-3, 20000.0, abi.GHOSTS_NONE)
    hard = np.load(OUT / "hard_r10_seed3.npz", allow_pickle=True)
    snap = {k[len("cells_"):]: hard[k] for k in hard.files if k.startswith("cells_")}
    solve_fixture("soft_on_hard_r10_seed3", abi.default_params(dt=3e-5, fixed_dt=1, seed=3, mode=abi.MODE_SOFT,
                                                               ghost_mode=abi.GHOSTS_SINGLE_RANK,
                                                               kcc=1333.3333333333333), snap, 3e-5)
    solve_fixture("hard_tight_r10_seed3", abi.default_params(dt=1e-3, fixed_dt=1, seed=3, mode=abi.MODE_HARD,
                                                             ghost_mode=abi.GHOSTS_SINGLE_RANK, tolerance=1e-6),
                  snap, 1e-3)
    snapshot_fixture("soft_r3_seed1", abi.MODE_SOFT, 1, 3.0, 3e-5, 1333.3333333333333, abi.GHOSTS_SINGLE_RANK)
    trajectory_fixture("traj_hard_seed3_3000", abi.MODE_HARD, 3, 3000, 1e-3, 20000.0, abi.GHOSTS_SINGLE_RANK, 1)
    trajectory_fixture("traj_hard_adaptive_seed5_2000", abi.MODE_HARD, 5, 2000, 1e-2, 20000.0,
                       abi.GHOSTS_SINGLE_RANK, 0)


if __name__ == "__main__":
    main()
