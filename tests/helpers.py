"""Shared helpers of the parity tests (fixtures, contact normalisation)."""
from __future__ import annotations

from pathlib import Path

import numpy as np

from pcc_b200 import abi

GOLDEN = Path(__file__).resolve().parent / "golden"


def load_fixture(name: str) -> dict:
    d = np.load(GOLDEN / f"{name}.npz", allow_pickle=True)
    return {k: d[k] for k in d.files}


def sub(fx: dict, prefix: str) -> dict:
    return {k[len(prefix):]: v for k, v in fx.items() if k.startswith(prefix)}


def params_of(fx: dict, **over) -> abi.Params:
    p = abi.default_params()
    for k, v in fx["params"][0].items():
        setattr(p, k, v)
    for k, v in over.items():
        setattr(p, "lambda_" if k == "lambda" else k, v)
    return p


def normalized_contacts(c: dict) -> dict:
    """Orient every contact as (smaller id, larger id) -- the reference's
    orientation follows hash-map iteration order -- and sort by ids, then by
    separation, so two lists of the same pairs line up entry by entry."""
    gi = np.asarray(c["gid_i"]).copy()
    gj = np.asarray(c["gid_j"]).copy()
    n = np.asarray(c["normal"]).reshape(-1, 3).copy()
    ri = np.asarray(c["r_i"]).reshape(-1, 3).copy()
    rj = np.asarray(c["r_j"]).reshape(-1, 3).copy()
    si = np.asarray(c["stress_i"]).copy()
    sj = np.asarray(c["stress_j"]).copy()
    swap = gi > gj
    gi[swap], gj[swap] = gj[swap], gi[swap].copy()
    n[swap] = -n[swap]
    ri[swap], rj[swap] = rj[swap], ri[swap].copy()
    si[swap], sj[swap] = sj[swap], si[swap].copy()
    out = {"gid_i": gi, "gid_j": gj, "normal": n, "r_i": ri, "r_j": rj, "stress_i": si, "stress_j": sj,
           "sd": np.asarray(c["sd"]).copy(), "gamma": np.asarray(c["gamma"]).copy(),
           "contact_point": np.asarray(c["contact_point"]).reshape(-1, 3).copy(),
           "phase": np.asarray(c["phase"]).copy()}
    order = np.lexsort((out["sd"], gj, gi))
    return {k: v[order] for k, v in out.items()}


def cells_max_diff(a: dict, b: dict, keys=("x", "y", "z", "q0", "q1", "q2", "q3", "length")) -> dict:
    return {k: float(np.max(np.abs(np.asarray(a[k], float) - np.asarray(b[k], float)))) if len(a[k]) else 0.0
            for k in keys}
