"""Brownian external velocity (temperature > 0) against the reference.

The reference adds, at ReLCP phase 0 of every hard step and at every soft
step, a rotational velocity T u1 u_k imp^3 per cell drawn from one
process-wide, default-seeded std::mt19937 (dynamics/Physics.cpp:19,59-81;
simulation/Particle.cpp:174-190): two draws per cell in a monolayer, four
otherwise.  The fixture (tests/golden/make_golden.py, brownian_r10_seed3)
holds two solver calls in a row on the same handle for each case, so the
second call checks that the device's generator continues the stream, and a
1,500-step trajectory from one cell.  Tolerances as in test_gpu_parity.py:
hard solves 1e-6 on positions, soft 1e-12.
"""
from __future__ import annotations

import numpy as np
import pytest

from helpers import cells_max_diff, load_fixture, sub
from pcc_b200 import abi
from pcc_b200.device import Colony

pytestmark = pytest.mark.gpu


def params_from(d) -> abi.Params:
    p = abi.default_params()
    for k, v in d.items():
        setattr(p, k, v)
    return p


@pytest.mark.parametrize("case,tol", [("hard_", 1e-6), ("hard3d_", 1e-6), ("soft_", 1e-12)])
def test_brownian_solves_match_reference(case, tol):
    fx = load_fixture("brownian_r10_seed3")
    p = params_from(fx[f"{case}params"][0])
    assert p.temperature > 0
    g = Colony(p)
    g.set_cells(sub(fx, "cells_"))
    for k in (1, 2):
        st = g.solve(p.dt, 0)
        want = fx[f"{case}solve{k}_stats"][0]
        d = cells_max_diff(g.get_cells(), sub(fx, f"{case}solve{k}_cells_"))
        print(f"\n{case}{k}: relcp {st['relcp_iterations']}/{want['relcp_iterations']} bbpgd "
              f"{st['bbpgd_iterations']}/{want['bbpgd_iterations']} positions within {max(d.values()):.3g}")
        assert st["n_constraints"] == want["n_constraints"]
        assert max(d.values()) < tol, (k, d)
    # the kicks are really there: the same call at temperature 0 moves the quaternions differently
    q = abi.Params.from_buffer_copy(p)
    q.temperature = 0.0
    g0 = Colony(q)
    g0.set_cells(sub(fx, "cells_"))
    g0.solve(p.dt, 0)
    d0 = cells_max_diff(g0.get_cells(), sub(fx, f"{case}solve1_cells_"), keys=("q0", "q1", "q2", "q3"))
    assert max(d0.values()) > 100 * tol, d0


def test_brownian_trajectory_matches_reference():
    fx = load_fixture("brownian_r10_seed3")
    p = params_from(fx["traj_params"][0])
    g = Colony(p)
    g.set_cells(abi.seed_cell(int(p.seed)))
    hist = [g.step() for _ in range(len(fx["traj_hist_n_cells"]))]
    np.testing.assert_array_equal([h["n_cells"] for h in hist], fx["traj_hist_n_cells"])
    d = cells_max_diff(g.get_cells(), sub(fx, "traj_final_"))
    assert max(d.values()) < 1e-6, d
