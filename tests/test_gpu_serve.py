"""Continuous batching of independent colonies (pcc_serve).

Each job grows one colony from a single cell.  Run one at a time and run four
at a time with staggered arrivals, every job must end bit-identically (same
steps, cells, BBPGD iterations and final-state checksum): jobs share nothing
on the device and no kernel result depends on timing.  Admission honours the
arrival order, the slot count and the HBM budget.
"""
from __future__ import annotations

import pytest

from pcc_b200 import abi
from pcc_b200.device import PccError, serve

pytestmark = pytest.mark.gpu


def make_jobs(arrival_step: float = 0.0):
    jobs = []
    for k in range(6):
        hard = k != 4
        p = abi.default_params(mode=abi.MODE_HARD if hard else abi.MODE_SOFT, seed=100 + k,
                               dt=1e-3 if hard else 1e-4, fixed_dt=0 if hard else 1, dt_cap=1e-3,
                               tau=1.0 / (0.6 + 0.15 * k), kcc=1333.3333333333333)
        jobs.append({"params": p, "end_radius": 2.0 + 0.5 * (k % 4) if hard else 1.0,
                     "arrival_s": k * arrival_step, "max_steps": 20000})
    return jobs


def test_jobs_identical_alone_and_in_the_mix():
    alone, _ = serve(make_jobs(), slots=1)
    mixed, wall = serve(make_jobs(arrival_step=0.02), slots=4)
    for a, b in zip(alone, mixed):
        for k in ("status", "steps", "cells", "bbpgd_iterations", "checksum", "cell_steps"):
            assert a[k] == b[k], (k, a, b)
        assert b["arrival_s"] <= b["start_s"] <= b["finish_s"] <= wall + 1e-6
    assert all(r["cells"] > 1 for r in alone)


def test_admission_respects_slots_and_budget():
    jobs = make_jobs()
    res, _ = serve(jobs, slots=2)
    # never more than two jobs in flight
    events = sorted([(r["start_s"], 1) for r in res] + [(r["finish_s"], -1) for r in res])
    live = peak = 0
    for _, d in events:
        live += d
        peak = max(peak, live)
    assert peak <= 2
    # a budget that fits one job at a time serialises them
    one = max(r["footprint_bytes"] for r in res)
    res1, _ = serve(jobs, slots=6, hbm_budget_bytes=one * 1.01)
    spans = sorted((r["start_s"], r["finish_s"]) for r in res1)
    assert all(spans[i][1] <= spans[i + 1][0] + 1e-3 for i in range(len(spans) - 1))
    # a job that can never fit is refused up front
    with pytest.raises(PccError):
        serve(jobs, slots=2, hbm_budget_bytes=one * 0.5)


def test_request_loop_accepts_jobs_while_running():
    """pcc_server: jobs submitted while others run are admitted as slots free
    up, and each finishes exactly as it does alone."""
    import time
    from pcc_b200.device import Server
    jobs = make_jobs()
    alone, _ = serve(jobs, slots=1)
    sv = Server(slots=3)
    ids = []
    for j in jobs:
        ids.append(sv.submit(j))
        time.sleep(0.05)
    got = {}
    deadline = time.time() + 600
    while len(got) < len(jobs) and time.time() < deadline:
        got.update(sv.poll(wait_s=1.0))
    q, r = sv.pending()
    sv.close()
    assert (q, r) == (0, 0) and sorted(got) == sorted(ids)
    for k, a in zip(ids, alone):
        b = got[k]
        for f in ("status", "steps", "cells", "bbpgd_iterations", "checksum"):
            assert a[f] == b[f], (f, a, b)
        assert b["arrival_s"] <= b["start_s"] <= b["finish_s"]


def test_batch_steps_every_colony_as_alone():
    """pcc_batch: four colonies stepped together (one context and stream each,
    a host thread pool) end exactly where each ends when stepped alone."""
    import numpy as np
    from pcc_b200.device import Batch, Colony
    # fixed dt: every colony has divided by step 1,000 (l grows by dt / tau per step)
    params = [abi.default_params(dt=1e-3, fixed_dt=1, seed=200 + k, tau=1.0 / (0.7 + 0.2 * k)) for k in range(4)]
    b = Batch(params)
    for k in range(4):
        b[k].set_cells(abi.seed_cell(200 + k))
    for _ in range(1500):
        stats = b.step()
    got = [b[k].get_cells() for k in range(4)]
    assert all(s["n_cells"] > 1 for s in stats)
    for k in range(4):
        g = Colony(params[k])
        g.set_cells(abi.seed_cell(200 + k))
        for _ in range(1500):
            g.step()
        want = g.get_cells()
        for f in ("x", "y", "q0", "q3", "length"):
            np.testing.assert_array_equal(got[k][f], want[f], err_msg=f)
    b.close()
