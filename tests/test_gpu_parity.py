"""Parity of the device library (through its C ABI) with the reference.

Inputs are the golden snapshots made by the reference's own code
(tests/golden/make_golden.py) and the plain-C oracle where a case is built on
the fly.  Tolerances, and why:
  * contact detection: bit-exact (same binning, same IEEE operations, no FMA);
  * soft model, one call: positions within 1e-12 absolute -- the per-cell
    force sums add the same terms in a different order;
  * hard model: the device reduces the BBPGD dot products in a different order
    (fixed-chunk trees instead of one sequential sum), so iterates differ by
    rounding and the solver may stop at a different multiple of 10
    iterations.  Both stop at residual <= tolerance, so positions agree to the
    solver tolerance: 1e-6 absolute after one call at tolerance 1e-3 (the
    iterates agree to rounding there), 2 x tolerance at tolerance 1e-6 (18,000
    BB iterations amplify rounding to the residual level), 5e-3 after 3000
    steps of growth (trajectories of a contact-driven colony are chaotic),
    and both runs satisfy the LCP (gamma >= 0, max overlap <= tolerance).
"""
from __future__ import annotations

import numpy as np
import pytest

from helpers import cells_max_diff, load_fixture, normalized_contacts, params_of, sub
from oracles import OracleColony
from pcc_b200 import abi
from pcc_b200.device import Colony, PccError

pytestmark = pytest.mark.gpu

SNAPSHOTS = ["hard_r10_seed3", "hard_r5_seed0_noghost", "soft_r3_seed1"]


@pytest.mark.parametrize("name", SNAPSHOTS)
@pytest.mark.parametrize("tag,tol", [("det25_", 0.25), ("dettol_", 1e-3), ("det0_", 0.0)])
def test_contacts_bit_exact(name, tag, tol):
    fx = load_fixture(name)
    g = Colony(params_of(fx))
    g.set_cells(sub(fx, "cells_"))
    got = normalized_contacts(g.detect(tol, 0))
    want = normalized_contacts(sub(fx, tag))
    assert got["gid_i"].size == want["gid_i"].size
    for k in want:
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)


def test_contacts_bit_exact_without_ghost_copies():
    fx = load_fixture("hard_r10_seed3")
    p = params_of(fx, ghost_mode=abi.GHOSTS_NONE)
    g, o = Colony(p), OracleColony(p)
    g.set_cells(sub(fx, "cells_"))
    o.set_cells(sub(fx, "cells_"))
    a, b = normalized_contacts(g.detect(0.25)), normalized_contacts(o.detect(0.25))
    for k in b:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    assert a["gid_i"].size < load_fixture("hard_r10_seed3")["det25_sd"].size  # ghosts add duplicates


def test_soft_solve_matches_reference():
    fx = load_fixture("soft_on_hard_r10_seed3")
    p = params_of(fx)
    g = Colony(p)
    g.set_cells(sub(fx, "cells_"))
    st = g.solve(p.dt, 0)
    want = fx["solve_stats"][0]
    assert st["n_constraints"] == want["n_constraints"]
    assert st["max_overlap"] == want["max_overlap"]
    got, ref = g.get_cells(), sub(fx, "solve_cells_")
    d = cells_max_diff(got, ref)
    assert max(d.values()) < 1e-12, d
    np.testing.assert_allclose(got["force"], ref["force"], rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(got["stress"], ref["stress"], rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(got["ldot"], ref["ldot"], rtol=1e-14)


@pytest.mark.parametrize("name,pos_tol", [("hard_r10_seed3", 1e-6), ("hard_tight_r10_seed3", 2e-6),
                                          ("hard_r5_seed0_noghost", 1e-6)])
def test_hard_solve_matches_reference(name, pos_tol):
    fx = load_fixture(name)
    p = params_of(fx)
    g = Colony(p)
    g.set_cells(sub(fx, "cells_"))
    st = g.solve(p.dt, 0)
    want = fx["solve_stats"][0]
    assert st["residual"] <= p.tolerance and st["max_overlap"] <= p.tolerance or st["relcp_iterations"] > 0
    assert abs(st["relcp_iterations"] - want["relcp_iterations"]) <= 1
    d = cells_max_diff(g.get_cells(), sub(fx, "solve_cells_"))
    assert max(d.values()) < pos_tol, (d, st, want)
    cons = g.constraints()
    assert np.all(cons["gamma"] >= 0.0)


def test_single_cell_growth_bit_exact_and_ten_iterations():
    p = abi.default_params(dt=1e-3, fixed_dt=1)
    g, o = Colony(p), OracleColony(p)
    g.set_cells(abi.seed_cell(0))
    o.set_cells(abi.seed_cell(0))
    for _ in range(700):
        sg, so = g.step(), o.step()
        assert sg["bbpgd_iterations"] == so["bbpgd_iterations"]
        assert sg["n_cells"] == so["n_cells"]
    assert sg["n_cells"] == 2
    d = cells_max_diff(g.get_cells(), o.get_cells())
    assert max(d.values()) == 0.0, d


def test_empty_colony_steps():
    g = Colony(abi.default_params(dt=1e-3, fixed_dt=1))
    g.set_cells({k: [] for k in abi.seed_cell(0)})
    st = g.step()
    assert st["n_cells"] == 0 and st["n_constraints"] == 0


def test_division_matches_oracle():
    """Five separated cells at division length: daughters, ages and draws
    follow the reference's divide (simulation/Particle.cpp:122-150)."""
    cells = {k: [] for k in abi.seed_cell(0)}
    for i in range(5):
        c = abi.seed_cell(100 + i)
        c["x"] = [10.0 * i]
        c["y"] = [3.0 * (i % 2)]
        c["length"] = [2.0]
        for k in cells:
            cells[k] += c[k]
    p = abi.default_params(dt=1e-3, fixed_dt=1, seed=42)
    g, o = Colony(p), OracleColony(p)
    g.set_cells(cells)
    o.set_cells(cells)
    sg, so = g.step(), o.step()
    assert sg["n_divided"] == so["n_divided"] == 5
    assert sg["n_cells"] == so["n_cells"] == 10
    a, b = g.get_cells(), o.get_cells()
    np.testing.assert_array_equal(a["age"], b["age"])
    d = cells_max_diff(a, b)
    assert max(d.values()) < 1e-12, d


def test_trajectory_matches_reference():
    fx = load_fixture("traj_hard_seed3_3000")
    p = params_of(fx)
    g = Colony(p)
    g.set_cells(sub(fx, "start_"))
    hist = [g.step() for _ in range(len(fx["hist_n_cells"]))]
    np.testing.assert_array_equal([h["n_cells"] for h in hist], fx["hist_n_cells"])
    assert all(h["max_overlap"] <= p.tolerance for h in hist)
    d = cells_max_diff(g.get_cells(), sub(fx, "final_"))
    assert max(d.values()) < 5e-3, d


def test_solve_is_deterministic():
    fx = load_fixture("hard_r10_seed3")
    p = params_of(fx)
    out = []
    for _ in range(2):
        g = Colony(p)
        g.set_cells(sub(fx, "cells_"))
        g.solve(p.dt, 0)
        out.append(g.get_cells())
    d = cells_max_diff(out[0], out[1], keys=("x", "y", "q0", "q3", "length", "ldot", "stress"))
    assert max(d.values()) == 0.0, d


@pytest.mark.parametrize("name", ["hard_r10_seed3", "hard_tight_r10_seed3"])
def test_planar_solver_bit_identical_to_general(name):
    """On a planar colony the packed 2D BBPGD kernel skips only exact zeros."""
    fx = load_fixture(name)
    out = []
    for variant in (abi.SOLVER_AUTO, abi.SOLVER_GENERAL):
        g = Colony(params_of(fx, solver_variant=variant))
        g.set_cells(sub(fx, "cells_"))
        st = g.solve(params_of(fx).dt, 0)
        out.append((st, g.get_cells(), g.constraints()))
    assert out[0][0] == out[1][0]
    for k in ("x", "y", "z", "q0", "q1", "q2", "q3", "length", "ldot", "stress", "impedance", "force", "velocity"):
        np.testing.assert_array_equal(out[0][1][k], out[1][1][k], err_msg=k)
    for k in ("gamma", "sd"):
        np.testing.assert_array_equal(out[0][2][k], out[1][2][k], err_msg=k)


def test_non_planar_colony_matches_oracle():
    """Cells tilted out of the plane take the general 3D path."""
    fx = load_fixture("hard_r5_seed0_noghost")
    cells = sub(fx, "cells_")
    rng = np.random.default_rng(0)
    n = len(cells["x"])
    cells["z"] = rng.uniform(-0.05, 0.05, n)
    tilt = rng.uniform(-0.05, 0.05, n)
    q = np.stack([cells["q0"], np.sin(tilt / 2) * cells["q0"], np.zeros(n), cells["q3"]], 1)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    cells["q0"], cells["q1"], cells["q2"], cells["q3"] = q.T
    p = params_of(fx)
    g, o = Colony(p), OracleColony(p)
    g.set_cells(cells)
    o.set_cells(cells)
    a, b = normalized_contacts(g.detect(0.25)), normalized_contacts(o.detect(0.25))
    for k in b:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    g.set_cells(cells)
    o.set_cells(cells)
    sg, so = g.solve(p.dt, 0), o.solve(p.dt, 0)
    assert sg["relcp_iterations"] == so["relcp_iterations"]
    d = cells_max_diff(g.get_cells(), o.get_cells())
    assert max(d.values()) < 1e-9, d
    assert np.max(np.abs(g.get_cells()["q1"])) > 0


def test_bbpgd_nonconvergence_raises_reference_message():
    fx = load_fixture("hard_r10_seed3")
    g = Colony(params_of(fx, max_bbpgd_iterations=5))
    g.set_cells(sub(fx, "cells_"))
    with pytest.raises(PccError, match="BBPGD did not converge") as e:
        g.solve(1e-3, 0)
    assert e.value.status == abi.PCC_ERR_NOCONV_BBPGD


def test_relcp_exhaustion_raises_reference_message():
    fx = load_fixture("hard_r10_seed3")
    g = Colony(params_of(fx, max_recursive_iterations=1))
    g.set_cells(sub(fx, "cells_"))
    with pytest.raises(PccError, match="Maximum number of constraint iterations reached") as e:
        g.solve(1e-3, 0)
    assert e.value.status == abi.PCC_ERR_NOCONV_RELCP


def _rows(c: dict) -> list:
    """Constraint rows as a sorted multiset of (phase, smaller id, larger id)."""
    a = np.minimum(c["gid_i"], c["gid_j"])
    b = np.maximum(c["gid_i"], c["gid_j"])
    return sorted(zip(np.asarray(c["phase"]).tolist(), a.tolist(), b.tolist()))


def test_later_relcp_phases_reuse_candidate_lists():
    """ReLCP phases after the first re-test the first phase's candidate lists
    instead of rebinning; every phase's constraint rows and the per-cell
    contact counts (Particle::num_constraints) are the reference's."""
    fx = load_fixture("hard_r10_seed3")
    p = params_of(fx)
    g = Colony(p)
    g.set_cells(sub(fx, "cells_"))
    g.profiling(False)
    st = g.solve(p.dt, 0)
    want = fx["solve_stats"][0]
    assert st["relcp_iterations"] == want["relcp_iterations"] == 4
    pr = g.profile()
    assert pr["detect_full_passes"] == 1 and pr["detect_list_passes"] == 4, pr
    assert _rows(g.constraints()) == _rows(sub(fx, "solve_cons_"))
    np.testing.assert_array_equal(g.get_cells()["num_constraints"], fx["solve_cells_num_constraints"])


@pytest.mark.parametrize("over", [{"tolerance": 0.3}, {"linked_cell_size": 1.95}])
def test_candidate_lists_fall_back_to_full_pass(over):
    """When the displacement bound cannot prove the lists complete (a later
    tolerance beyond the list reach; bins shorter than the longest cell plus
    the reach) every phase rebins, and the result is the oracle's."""
    fx = load_fixture("hard_r10_seed3")
    p = params_of(fx, **over)
    g, o = Colony(p), OracleColony(p)
    g.set_cells(sub(fx, "cells_"))
    o.set_cells(sub(fx, "cells_"))
    g.profiling(False)
    sg, so = g.solve(p.dt, 0), o.solve(p.dt, 0)
    pr = g.profile()
    assert pr["detect_list_passes"] == 0 and pr["detect_full_passes"] == sg["relcp_iterations"] + 1, pr
    assert sg["relcp_iterations"] == so["relcp_iterations"]
    assert _rows(g.constraints()) == _rows(o.constraints())
    np.testing.assert_array_equal(g.get_cells()["num_constraints"], o.get_cells()["num_constraints"])
    d = cells_max_diff(g.get_cells(), o.get_cells())
    assert max(d.values()) < 1e-6, d


@pytest.mark.parametrize("name", ["soft_on_hard_r10_seed3", "soft_r3_seed1", "hard_r5_seed0_noghost"])
def test_num_constraints_match_reference(name):
    """Particle::num_constraints after one call, including the counts a cell
    with a self-ghost loses to its copy."""
    fx = load_fixture(name)
    p = params_of(fx)
    g = Colony(p)
    g.set_cells(sub(fx, "cells_"))
    g.solve(p.dt, 0)
    np.testing.assert_array_equal(g.get_cells()["num_constraints"], fx["solve_cells_num_constraints"])


@pytest.mark.parametrize("name", ["hard_r10_seed3", "hard_tight_r10_seed3"])
def test_mixed_precision_solve_close_to_fp64(name):
    """Mixed precision (FP32 D, L, M, U; FP64 gamma, BB dots, residual) meets
    the same LCP tolerance.  FP32 rounding sends the Barzilai-Borwein iterates
    down a different path, which stops at another point of the residual <= tol
    set, so cells agree with the FP64 path to the solver tolerance (twice tol,
    plus rounding), not to rounding."""
    fx = load_fixture(name)
    out = []
    for prec in (abi.PRECISION_FP64, abi.PRECISION_MIXED):
        p = params_of(fx, precision=prec)
        g = Colony(p)
        g.set_cells(sub(fx, "cells_"))
        st = g.solve(p.dt, 0)
        out.append((st, g.get_cells(), g.constraints()))
    (s64, c64, k64), (s32, c32, k32) = out
    tol = params_of(fx).tolerance
    assert s32["residual"] <= tol and s32["max_overlap"] <= tol
    assert np.all(k32["gamma"] >= 0.0)
    d = cells_max_diff(c64, c32)
    assert max(d.values()) < 2 * tol + 1e-6, d
    assert s32["bbpgd_iterations"] > 0


def test_mixed_precision_trajectory_matches_reference():
    """3000 steps from one cell: the growth rates feel the FP32 rounding through
    the contact stresses, so a division may come a few steps earlier or later
    than in the reference; the colony divides the same number of times, each
    within 50 steps of the reference, and every step meets the tolerance."""
    fx = load_fixture("traj_hard_seed3_3000")
    p = params_of(fx, precision=abi.PRECISION_MIXED)
    g = Colony(p)
    g.set_cells(sub(fx, "start_"))
    hist = [g.step() for _ in range(len(fx["hist_n_cells"]))]
    got = np.array([h["n_cells"] for h in hist])
    want = np.asarray(fx["hist_n_cells"])
    assert got[-1] == want[-1]
    for k in range(int(want[0]) + 1, int(want[-1]) + 1):
        assert abs(int(np.argmax(got >= k)) - int(np.argmax(want >= k))) <= 50, k
    assert all(h["max_overlap"] <= p.tolerance for h in hist)


def test_one_cta_solver_bit_identical_to_multi_block():
    """A planar colony of ~800 cells and a few thousand constraints solves in
    the one-CTA kernel (four 256-thread groups own the chunks, named-barrier
    reductions); the 3D kernel runs the same solve in one 256-thread block and,
    once the accumulated constraints outgrow it, over a grid of blocks.  Same
    chunks, same reduction trees: the results agree bit for bit."""
    from pcc_b200 import synth
    cells = synth.dense_colony(16.0, seed=1, lane_gap=0.0, end_gap=0.0)
    out = []
    for variant in (abi.SOLVER_AUTO, abi.SOLVER_GENERAL):
        p = abi.default_params(dt=3e-4, fixed_dt=1, solver_variant=variant)
        g = Colony(p)
        g.set_cells(cells)
        st = g.solve(p.dt, 1)
        out.append((st, g.get_cells(), g.constraints()))
    assert len(cells["x"]) <= 1024 and out[0][0]["n_constraints"] > 2 * 1024
    assert out[0][0] == out[1][0]
    for k in ("x", "y", "q0", "q3", "length", "ldot", "stress", "force", "velocity"):
        np.testing.assert_array_equal(out[0][1][k], out[1][1][k], err_msg=k)
    np.testing.assert_array_equal(out[0][2]["gamma"], out[1][2]["gamma"])
