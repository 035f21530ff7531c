"""The CPU oracle (plain-C restatement, oracle/pcc_oracle.c) pinned against the
reference's own outputs.

Golden fixtures in tests/golden/ were produced by the reference simulator's
sources compiled in place (tests/golden/make_golden.py).  Both builds are
IEEE-strict, so the restatement must reproduce them bit for bit: contact lists
(after orienting each pair by id), one solver call, multi-step trajectories
and the division draws.
"""
from __future__ import annotations

import numpy as np
import pytest

from helpers import cells_max_diff, load_fixture, normalized_contacts, params_of, sub
from oracles import OracleColony, oracle_division_length

SNAPSHOTS = ["hard_r10_seed3", "hard_r5_seed0_noghost", "soft_r3_seed1"]


def test_division_draws_match_libstdcxx():
    fx = load_fixture("division_draws")
    for seed, k, L, v in zip(fx["seed"], fx["k"], fx["length"], fx["value"]):
        assert oracle_division_length(int(seed), int(k), float(L)) == v


@pytest.mark.parametrize("name", SNAPSHOTS)
@pytest.mark.parametrize("tag,tol", [("det25_", 0.25), ("dettol_", 1e-3), ("det0_", 0.0)])
def test_contacts_bit_exact(name, tag, tol):
    fx = load_fixture(name)
    o = OracleColony(params_of(fx))
    o.set_cells(sub(fx, "cells_"))
    got = normalized_contacts(o.detect(tol, 0))
    want = normalized_contacts(sub(fx, tag))
    assert got["gid_i"].size == want["gid_i"].size
    for k in want:
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)


@pytest.mark.parametrize("name", SNAPSHOTS + ["soft_on_hard_r10_seed3", "hard_tight_r10_seed3"])
def test_one_solve_bit_exact(name):
    fx = load_fixture(name)
    p = params_of(fx)
    o = OracleColony(p)
    o.set_cells(sub(fx, "cells_"))
    st = o.solve(p.dt, 0)
    want = fx["solve_stats"][0]
    for k in ("relcp_iterations", "bbpgd_iterations", "residual", "max_overlap", "n_constraints", "n_cells"):
        assert st[k] == want[k], k
    got = o.get_cells()
    ref = sub(fx, "solve_cells_")
    for k in ("x", "y", "z", "q0", "q1", "q2", "q3", "length", "ldot", "impedance", "stress", "force", "velocity",
              "num_constraints"):
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    gc = normalized_contacts(o.constraints())
    rc = normalized_contacts(sub(fx, "solve_cons_"))
    for k in rc:
        np.testing.assert_array_equal(gc[k], rc[k], err_msg=k)


@pytest.mark.parametrize("name", ["traj_hard_seed3_3000", "traj_hard_adaptive_seed5_2000"])
def test_trajectory_bit_exact(name):
    fx = load_fixture(name)
    p = params_of(fx)
    o = OracleColony(p)
    o.set_cells(sub(fx, "start_"))
    hist = [o.step() for _ in range(len(fx["hist_n_cells"]))]
    for k in ("n_cells", "bbpgd_iterations", "relcp_iterations", "n_constraints", "residual", "max_overlap",
              "dt_used", "colony_radius", "n_divided"):
        np.testing.assert_array_equal(np.array([h[k] for h in hist]), fx[f"hist_{k}"], err_msg=k)
    d = cells_max_diff(o.get_cells(), sub(fx, "final_"))
    assert all(v == 0.0 for v in d.values()), d


def test_single_cell_reports_ten_bbpgd_iterations():
    """Empty constraint set: res0 = 0, the first residual check at iteration 10
    passes (solver/BBPGD.cpp:64-80)."""
    from pcc_b200 import abi
    o = OracleColony(abi.default_params(dt=1e-3, fixed_dt=1))
    o.set_cells(abi.seed_cell(0))
    st = o.step()
    assert st["bbpgd_iterations"] == 10 and st["relcp_iterations"] == 1 and st["n_constraints"] == 0


def test_isolated_cell_divides_after_694_steps():
    """l_{n+1} = l_n (1 + dt/tau) reaches 2 l0 after ceil(ln 2 / ln 1.001) = 694 steps."""
    from pcc_b200 import abi
    o = OracleColony(abi.default_params(dt=1e-3, fixed_dt=1))
    o.set_cells(abi.seed_cell(0))
    n = [o.step()["n_cells"] for _ in range(700)]
    assert n.index(2) == 694


def test_nonconvergence_is_reported():
    from pcc_b200 import abi
    fx = load_fixture("hard_r10_seed3")
    o = OracleColony(params_of(fx, max_bbpgd_iterations=5))
    o.set_cells(sub(fx, "cells_"))
    with pytest.raises(RuntimeError, match="BBPGD did not converge"):
        o.solve(1e-3, 0)
    o = OracleColony(params_of(fx, max_recursive_iterations=1))
    o.set_cells(sub(fx, "cells_"))
    with pytest.raises(RuntimeError, match="Maximum number of constraint iterations"):
        o.solve(1e-3, 0)
