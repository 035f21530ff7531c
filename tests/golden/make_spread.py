"""Measures how far the reference's own whole runs spread when only the
division draws change: the config-0 (hard, dt = 1e-3) and config-1 (soft,
dt = 3e-5) runs of grown_hard_r20_seed0 / grown_soft_r20_seed0 repeated with
division streams 1..K (the first cell's orientation unchanged), each grown to
R = 20 by the reference's own code (oracle/_ref/libpccref_strict.so).  A
whole run is chaotic once contacts matter, so a device run is compared with
the reference's run within this spread.

Run from the repository root (reference build present):
    python tests/golden/make_spread.py [K]
Writes spread_r20.npz: per mode, steps to R = 20, final cell count and the
cell count every 100 steps of each run.
"""
from __future__ import annotations

import multiprocessing as mp
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
OUT = Path(__file__).resolve().parent


def one_run(args):
    mode, seed = args
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    import pcc_pkg
    pcc_pkg.load_package()
    from pcc_b200 import abi
    from oracles import RefColony
    if mode == "hard":
        p = abi.default_params(dt=1e-3, fixed_dt=1, seed=seed, mode=abi.MODE_HARD, ghost_mode=abi.GHOSTS_SINGLE_RANK)
    else:
        p = abi.default_params(dt=3e-5, fixed_dt=1, seed=seed, mode=abi.MODE_SOFT, ghost_mode=abi.GHOSTS_SINGLE_RANK,
                               kcc=1333.3333333333333)
    r = RefColony(p)
    r.set_cells(abi.seed_cell(0))
    n = []
    while r.colony_radius < 20.0 and len(n) < 10**7:
        n.append(r.step()["n_cells"])
    return mode, seed, len(n), n[-1], np.array(n[::100], np.int32)


def main(k: int):
    jobs = [(m, s) for m in ("hard", "soft") for s in range(1, k + 1)]
    with mp.get_context("spawn").Pool(min(len(jobs), max(1, mp.cpu_count() - 1))) as pool:
        res = pool.map(one_run, jobs, chunksize=1)
    out = {}
    for mode in ("hard", "soft"):
        rs = sorted((r for r in res if r[0] == mode), key=lambda r: r[1])
        out[f"{mode}_seeds"] = np.array([r[1] for r in rs])
        out[f"{mode}_steps"] = np.array([r[2] for r in rs])
        out[f"{mode}_final_cells"] = np.array([r[3] for r in rs])
        w = max(len(r[4]) for r in rs)
        out[f"{mode}_n_every_100"] = np.array([np.pad(r[4], (0, w - len(r[4])), constant_values=-1) for r in rs])
        print(mode, "steps", out[f"{mode}_steps"].tolist(), "cells", out[f"{mode}_final_cells"].tolist())
    np.savez_compressed(OUT / "spread_r20.npz", **out)


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else 3)
