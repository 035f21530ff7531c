"""Parity with the reference at colony sizes that run the multi-block solver.

Every fixture here was made by the reference's own code (tests/golden/make_golden.py):
  * grown_hard_r20_seed0 -- config 0 as the reference runs it: hard model,
    FP64, dt = 1e-3 fixed, grown from one cell (orientation from seed 0) to
    R = 20 (8,157 steps, 1,594 cells); snapshots at the first state past
    1,100 cells and at the end, each with contact lists, one solver call
    and a 10-step continuation;
  * dense_r20_seed0 / dense_r40_seed0 -- the benchmark's synthetic dense
    colony (1,308 / 5,280 cells, neighbours touching): contact lists, one
    hard and one soft solver call, a few steps with CFL-adaptive dt;
  * grown_soft_r20_seed0 -- config 1: soft model, dt = 3e-5, kcc = 4/3 E
    (E = 1e3, R_eff = 0.125), grown from one cell to R = 20.
Colonies above 1,024 cells run the multi-block cooperative BBPGD kernels
(k_bbpgd_planar<double> for FP64, <float> for mixed precision); each solve
test asserts that they did.

Tolerances, and why:
  * contact lists: bit-exact (same binning and IEEE operations); contacts
    within 1e-9 of the detection cutoff are counted separately and their
    count must match too;
  * one hard solver call at the reference's tolerance (1e-3): the device
    sums the BB dot products in another order, and over hundreds of
    Barzilai-Borwein iterations the iterates part from the reference's
    (the method is not monotone), so the two solvers can stop at different
    multiples of 10 iterations at two different points of the set where the
    projected residual is below the tolerance.  Such points differ by up to
    about the tolerance, so positions are required within 2 x tolerance,
    both results must satisfy the LCP (gamma >= 0, residual and max overlap
    <= tol, complementarity max |gamma_i phi_i| <= tol * max gamma, reported
    beside the reference's) and the ReLCP counts within one phase; the
    gamma and force differences are reported.  The same snapshot solved at
    tolerance 1e-6 pins the solve itself: there both land on the same
    positions within 10 x 1e-6.  gamma is not bounded there: a pair that
    is constrained again in a later ReLCP phase adds a linearly dependent
    row, so the LCP fixes the velocities (and positions) but not how the
    impulse is shared among the rows; its difference is reported;
  * soft model, one call: 1e-12 (force sums in another order);
  * steps: the x-sort renumbers cells every step, so after solves that
    differ at the tolerance level cells are matched by position (nearest
    cell) before comparing; a cell within rounding of the division length
    can divide a step earlier or later in one run than in the other, which
    moves its daughters by about a quarter of a cell length, so the cells of
    one such division are allowed that offset;
  * whole runs: contact-driven growth is chaotic, so whole runs are compared
    by their step counts and cell counts against the spread of the
    reference's own runs when only the division draws change
    (tests/golden/make_spread.py, spread_r20.npz).
"""
from __future__ import annotations

import numpy as np
import pytest

from helpers import cells_max_diff, load_fixture, normalized_contacts, params_of, sub
from pcc_b200 import abi
from pcc_b200.device import Colony

pytestmark = pytest.mark.gpu

BAND = 1e-9


def cutoff_band(c: dict, tol: float) -> int:
    return int(np.sum(np.abs(np.asarray(c["sd"]) - tol) < BAND))


def oriented_rows(c: dict) -> dict:
    """gid_i < gid_j on every row, rows sorted by ids then phi (gamma and phi
    do not depend on the orientation)."""
    gi, gj = np.asarray(c["gid_i"]).copy(), np.asarray(c["gid_j"]).copy()
    swap = gi > gj
    gi[swap], gj[swap] = gj[swap], gi[swap].copy()
    sd, g, ph = np.asarray(c["sd"]), np.asarray(c["gamma"]), np.asarray(c["phase"])
    o = np.lexsort((sd, gj, gi))
    return {"gid_i": gi[o], "gid_j": gj[o], "sd": sd[o], "gamma": g[o], "phase": ph[o]}


def complementarity(cons: dict) -> float:
    """max_i |gamma_i phi_i| over the returned constraint set."""
    g, phi = np.asarray(cons["gamma"]), np.asarray(cons["sd"])
    return float(np.max(np.abs(g * phi))) if g.size else 0.0


def matched_distances(a: dict, b: dict) -> np.ndarray:
    """Distance from each cell of `a` to the nearest cell of `b` (ids may be
    permuted by the x-sort)."""
    from scipy.spatial import cKDTree
    pa = np.stack([a["x"], a["y"], a["z"]], 1)
    pb = np.stack([b["x"], b["y"], b["z"]], 1)
    d, _ = cKDTree(pb).query(pa)
    return d


def matched_distance(a: dict, b: dict) -> float:
    """Largest distance from a cell of `a` to the nearest cell of `b`."""
    return float(matched_distances(a, b).max())


def within_reference_spread(what: str, got: float, ref: float, others: np.ndarray) -> tuple[float, float]:
    """The reference's run (`ref`) and its runs with other division draws
    (`others`) as one sample of n runs: `got` must lie in the 99 % prediction
    interval of one more run, mean +- t(0.995, n - 1) s sqrt(1 + 1/n) (s the
    sample standard deviation).  Returns (mean, half width)."""
    from scipy.stats import t as student_t
    runs = np.concatenate([[float(ref)], np.asarray(others, float)])
    n = runs.size
    mean, sd = float(runs.mean()), float(runs.std(ddof=1))
    half = float(student_t.ppf(0.995, n - 1)) * sd * np.sqrt(1.0 + 1.0 / n)
    print(f"{what}: {got} against the reference's {ref} and {sorted(np.asarray(others).tolist())} "
          f"(mean {mean:.1f}, sd {sd:.1f}; 99 % prediction interval +-{half:.1f}, got {got - mean:+.1f})")
    assert abs(got - mean) <= half, (what, got, mean, half)
    return mean, half


def check_contacts(fx: dict, prefix: str, tag: str, tol: float):
    p = params_of(fx)
    g = Colony(p)
    g.set_cells(sub(fx, f"{prefix}cells_"))
    got = normalized_contacts(g.detect(tol, 0))
    want = normalized_contacts(sub(fx, f"{prefix}{tag}"))
    assert got["gid_i"].size == want["gid_i"].size
    assert cutoff_band(got, tol) == cutoff_band(want, tol)
    for k in want:
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)
    return got["gid_i"].size, cutoff_band(got, tol)


def check_hard_solve(p: abi.Params, cells: dict, dt: float, want_stats: dict, want_cells: dict, want_cons: dict,
                     precision: int, pos_factor: float = 2.0):
    p = abi.Params.from_buffer_copy(p)
    p.precision = precision
    g = Colony(p)
    g.set_cells(cells)
    g.profiling(True)
    st = g.solve(dt, 0)
    prof = g.profile()
    assert prof["bbpgd_grid_launches"] >= 1 and prof["bbpgd_cta_launches"] == 0, prof
    tol = p.tolerance
    assert st["residual"] <= tol and st["max_overlap"] <= tol
    assert abs(st["relcp_iterations"] - want_stats["relcp_iterations"]) <= 1
    got_cells, got_cons = g.get_cells(), g.constraints()
    fp64 = precision == abi.PRECISION_FP64
    d = cells_max_diff(got_cells, want_cells)
    fscale = max(np.max(np.abs(want_cells["force"])), 1e-300)
    ferr = float(np.max(np.abs(got_cells["force"] - want_cells["force"]))) / fscale
    # gamma of the phase-0 rows: the same pairs on both sides (bit-exact detection)
    a, b = oriented_rows(got_cons), oriented_rows(want_cons)
    ra, rb = a["phase"] == 0, b["phase"] == 0
    assert ra.sum() == rb.sum()
    np.testing.assert_array_equal(a["gid_i"][ra], b["gid_i"][rb])
    np.testing.assert_array_equal(a["gid_j"][ra], b["gid_j"][rb])
    gscale = max(np.max(b["gamma"][rb]), 1e-300)
    gerr = float(np.max(np.abs(a["gamma"][ra] - b["gamma"][rb]))) / gscale
    comp, comp_ref = complementarity(got_cons), complementarity(want_cons)
    print(f"\n[{'fp64' if fp64 else 'mixed'}] n={len(cells['x'])} constraints={st['n_constraints']} "
          f"relcp={st['relcp_iterations']}/{want_stats['relcp_iterations']} "
          f"bbpgd={st['bbpgd_iterations']}/{want_stats['bbpgd_iterations']} pos={max(d.values()):.3g} "
          f"gamma_rel={gerr:.3g} force_rel={ferr:.3g} complementarity={comp:.3g} (reference {comp_ref:.3g})")
    assert max(d.values()) < pos_factor * tol, (d, st, want_stats)
    assert np.all(got_cons["gamma"] >= 0.0)
    assert comp <= tol * max(np.max(got_cons["gamma"]), 1.0), (comp, comp_ref)
    return max(d.values()), gerr, ferr


# ---------------------------------------------------------------- config 0 grown colony

@pytest.mark.parametrize("snap", ["mid_", "end_"])
@pytest.mark.parametrize("tag,tol", [("det25_", 0.25), ("dettol_", 1e-3), ("det0_", 0.0)])
def test_grown_colony_contacts_bit_exact(snap, tag, tol):
    fx = load_fixture("grown_hard_r20_seed0")
    n, band = check_contacts(fx, snap, tag, tol)
    print(f"\n{snap}{tag}: {n} contacts, {band} within {BAND:g} of the cutoff")


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
@pytest.mark.parametrize("snap", ["mid_", "end_"])
def test_grown_colony_solve_matches_reference(snap, precision):
    fx = load_fixture("grown_hard_r20_seed0")
    cells = sub(fx, f"{snap}cells_")
    assert len(cells["x"]) > 1024
    check_hard_solve(params_of(fx), cells, float(fx[f"{snap}dt"]), fx[f"{snap}solve_stats"][0],
                     sub(fx, f"{snap}solve_cells_"), sub(fx, f"{snap}solve_cons_"), precision)


def test_grown_colony_tight_solve_matches_reference():
    """The 1,100-cell snapshot at tolerance 1e-6 (FP64): both solvers converge
    to the same LCP solution."""
    fx = load_fixture("grown_hard_r20_tight")
    p = params_of(fx)
    assert p.tolerance == 1e-6
    pos, gerr, ferr = check_hard_solve(p, sub(fx, "cells_"), float(fx["dt"]), fx["solve_stats"][0],
                                       sub(fx, "solve_cells_"), sub(fx, "solve_cons_"), abi.PRECISION_FP64,
                                       pos_factor=10.0)


@pytest.mark.parametrize("name,prefix", [("dense_r40_seed0", ""), ("grown_hard_r20_seed0", "end_")])
def test_multi_block_planar_solver_bit_identical_to_general(name, prefix):
    """Above 1,024 cells the planar solve runs the multi-block kernel, whose
    warps draw cell units from counters and whose blocks each reduce the
    chunk partials themselves; the general 3D kernel runs the same chunks and
    per-cell sums with a static cell order and one reducing block.  Two planar
    solves and the general one give the same bits."""
    fx = load_fixture(name)
    cells = sub(fx, f"{prefix}cells_")
    dt = float(fx[f"{prefix}dt"]) if f"{prefix}dt" in fx else float(params_of(fx).dt)
    out = []
    for variant in (abi.SOLVER_AUTO, abi.SOLVER_AUTO, abi.SOLVER_GENERAL):
        g = Colony(params_of(fx, solver_variant=variant))
        g.set_cells(cells)
        g.profiling(True)
        st = g.solve(dt, 0)
        prof = g.profile()
        assert prof["bbpgd_grid_launches"] >= 1 and prof["bbpgd_cta_launches"] == 0, prof
        out.append((st, g.get_cells(), g.constraints()))
    assert len(cells["x"]) > 1024
    print(f"\n{name}: {out[0][0]['bbpgd_iterations']} iterations, {out[0][0]['relcp_iterations']} phases")
    for other in out[1:]:
        assert other[0] == out[0][0]
        for k in ("x", "y", "z", "q0", "q3", "length", "ldot", "stress", "impedance", "force", "velocity"):
            np.testing.assert_array_equal(other[1][k], out[0][1][k], err_msg=k)
        for k in ("gamma", "sd"):
            np.testing.assert_array_equal(other[2][k], out[0][2][k], err_msg=k)


@pytest.mark.parametrize("snap", ["mid_", "end_"])
def test_grown_colony_continuation_matches_reference(snap):
    """Ten full steps (divide, x-sort, ReLCP, move, grow) from each snapshot."""
    fx = load_fixture("grown_hard_r20_seed0")
    p = params_of(fx)
    g = Colony(p)
    g.set_cells(sub(fx, f"{snap}cells_"))
    g.dt = float(fx[f"{snap}dt"])
    hist = [g.step() for _ in range(len(fx[f"{snap}cont_hist_n_cells"]))]
    final = g.get_cells()
    want = sub(fx, f"{snap}cont_final_")
    # both directions: a division that happened in one run only leaves its two
    # daughters (in that run) and its undivided parent (in the other) unmatched
    d = np.concatenate([matched_distances(final, want), matched_distances(want, final)])
    near = 10 * 2 * p.tolerance
    far = d[d >= near]
    print(f"\n{snap}: 10 steps, {d.size - far.size} of {d.size} cells within {near:g} of a cell of the other "
          f"run, the rest within {d.max():.3g}")
    # a division can land one step apart (lengths differ at the rounding level)
    got_n = np.array([h["n_cells"] for h in hist])
    assert np.max(np.abs(got_n - fx[f"{snap}cont_hist_n_cells"])) <= 1
    assert abs(int(got_n[-1]) - int(fx[f"{snap}cont_hist_n_cells"][-1])) <= 1
    assert all(h["max_overlap"] <= p.tolerance for h in hist)
    # at most one division on a different cell: the two daughters and the
    # undivided cell on each side (6 unmatched), each about a quarter of the
    # dividing cell's length from its nearest counterpart
    assert far.size <= 6, far
    assert d.max() < 0.4 * float(np.max(final["length"])), d.max()


def test_grown_colony_from_one_cell():
    """Config 0 end to end: 8,157 steps from one cell to R = 20 on the device,
    against the reference's own run.  Growth is identical until contacts
    matter, after which rounding differences in the solver make the
    trajectories part (division waves shift by a step or two); once the
    colony has 200 cells the counts must stay within 10 % of the reference's
    at every step, and the step count to R = 20 and the cell count there
    must lie in the 99 % prediction interval of the reference's own runs
    (this one and six with other division draws)."""
    fx = load_fixture("grown_hard_r20_seed0")
    p = params_of(fx)
    g = Colony(p)
    g.set_cells(abi.seed_cell(int(p.seed)))
    want = fx["hist_n_cells"]
    got = []
    radius = 0.0
    while radius < 20.0 and len(got) < int(len(want) * 1.05):
        st = g.step()
        got.append(st["n_cells"])
        radius = st["colony_radius"]
        assert st["max_overlap"] <= p.tolerance
    got = np.array(got)
    k = min(len(got), len(want))
    first_diff = int(np.argmax(got[:k] != want[:k])) if np.any(got[:k] != want[:k]) else k
    rel = np.abs(got[:k] - want[:k]) / want[:k]
    print(f"\nsteps {len(got)} (reference {len(want)}), cells {got[-1]} (reference {want[-1]}), "
          f"identical cell counts through step {first_diff}, largest relative difference {rel.max():.3g}")
    assert radius >= 20.0
    spread = load_fixture("spread_r20")
    within_reference_spread("steps to R = 20", len(got), len(want), spread["hard_steps"])
    within_reference_spread("cells at R = 20", int(got[-1]), int(want[-1]), spread["hard_final_cells"])
    # identical growth until contacts matter (the division draws are the same)
    assert first_diff >= 2000
    big = want[:k] >= 200
    assert rel[big].max() <= 0.10


# ---------------------------------------------------------------- dense synthetic colonies

@pytest.mark.parametrize("name,tag,tol", [("dense_r20_seed0", "det25_", 0.25), ("dense_r20_seed0", "dettol_", 1e-3),
                                          ("dense_r20_seed0", "det0_", 0.0), ("dense_r40_seed0", "det25_", 0.25)])
def test_dense_colony_contacts_bit_exact(name, tag, tol):
    n, band = check_contacts(load_fixture(name), "", tag, tol)
    print(f"\n{name} {tag}: {n} contacts, {band} within {BAND:g} of the cutoff")


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
@pytest.mark.parametrize("name", ["dense_r20_seed0", "dense_r40_seed0"])
def test_dense_colony_solve_matches_reference(name, precision):
    fx = load_fixture(name)
    p = params_of(fx)
    check_hard_solve(p, sub(fx, "cells_"), p.dt, fx["solve_stats"][0], sub(fx, "solve_cells_"),
                     sub(fx, "solve_cons_"), precision)


@pytest.mark.parametrize("name", ["dense_r20_seed0", "dense_r40_seed0"])
def test_dense_colony_soft_solve_matches_reference(name):
    fx = load_fixture(name)
    p = abi.default_params()
    for k, v in fx["soft_params"][0].items():
        setattr(p, k, v)
    g = Colony(p)
    g.set_cells(sub(fx, "cells_"))
    st = g.solve(p.dt, 0)
    want, ref = fx["soft_solve_stats"][0], sub(fx, "soft_solve_cells_")
    assert st["n_constraints"] == want["n_constraints"]
    got = g.get_cells()
    d = cells_max_diff(got, ref)
    assert max(d.values()) < 1e-12, d
    np.testing.assert_allclose(got["force"], ref["force"], rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(got["stress"], ref["stress"], rtol=1e-12, atol=1e-9)


@pytest.mark.parametrize("name", ["dense_r20_seed0", "dense_r40_seed0"])
def test_dense_colony_adaptive_steps_match_reference(name):
    """Full steps with CFL-adaptive dt (capped at 1e-3) from the packing."""
    fx = load_fixture(name)
    p = params_of(fx)
    g = Colony(p)
    g.set_cells(sub(fx, "cells_"))
    hist = [g.step() for _ in range(len(fx["cont_hist_n_cells"]))]
    d = matched_distance(g.get_cells(), sub(fx, "cont_final_"))
    dt_rel = np.max(np.abs(np.array([h["dt_used"] for h in hist]) - fx["cont_hist_dt_used"]) / fx["cont_hist_dt_used"])
    print(f"\n{name}: {len(hist)} adaptive steps, every cell within {d:.3g} of a reference cell, "
          f"dt within {dt_rel:.3g} relative")
    np.testing.assert_array_equal([h["n_cells"] for h in hist], fx["cont_hist_n_cells"])
    assert dt_rel < 1e-3
    np.testing.assert_allclose([h["colony_radius"] for h in hist], fx["cont_hist_colony_radius"], rtol=1e-4)
    assert d < len(hist) * 2 * p.tolerance, d


# ---------------------------------------------------------------- adaptive dt, soft growth

def test_adaptive_dt_trajectory_matches_reference():
    """2,000 steps from one cell with Domain::adaptDt (no fixed dt): the dt
    history follows the reference's and the cell counts are identical."""
    fx = load_fixture("traj_hard_adaptive_seed5_2000")
    p = params_of(fx)
    assert p.fixed_dt == 0
    g = Colony(p)
    g.set_cells(sub(fx, "start_"))
    hist = [g.step() for _ in range(len(fx["hist_n_cells"]))]
    dts = np.array([h["dt_used"] for h in hist])
    rel = np.abs(dts - fx["hist_dt_used"]) / fx["hist_dt_used"]
    d = cells_max_diff(g.get_cells(), sub(fx, "final_"))
    print(f"\nadaptive dt: largest relative dt difference {rel.max():.3g} over {len(dts)} steps, "
          f"positions within {max(d.values()):.3g}")
    np.testing.assert_array_equal([h["n_cells"] for h in hist], fx["hist_n_cells"])
    assert rel.max() < 1e-3
    assert max(d.values()) < 5e-3, d


def test_soft_colony_grown_to_r20():
    """Config 1 end to end: the soft model from one cell to R = 20 at
    dt = 3e-5 on the device, against the spread of the reference's runs
    (steps and cells at R = 20); then one force assembly on the reference's
    final state."""
    fx = load_fixture("grown_soft_r20_seed0")
    p = params_of(fx)
    want = fx["hist_n_cells"]
    g = Colony(p)
    g.set_cells(abi.seed_cell(int(p.seed)))
    steps, cs, st = g.run(20.0, int(len(want) * 1.05))
    print(f"\nsoft: {steps} steps (reference {len(want)}), {st['n_cells']} cells (reference {want[-1]})")
    assert st["colony_radius"] >= 20.0
    spread = load_fixture("spread_r20")
    within_reference_spread("soft steps to R = 20", steps, len(want), spread["soft_steps"])
    within_reference_spread("soft cells at R = 20", int(st["n_cells"]), int(want[-1]), spread["soft_final_cells"])
    g = Colony(p)
    g.set_cells(sub(fx, "end_cells_"))
    g.solve(p.dt, 0)
    d = cells_max_diff(g.get_cells(), sub(fx, "end_solve_cells_"))
    assert max(d.values()) < 1e-12, d
