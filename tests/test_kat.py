"""Known-answer tests of the pinned oracle: hand-derived contact geometry and
a two-cell LCP with a closed-form solution, checked against the plain-C
restatement and the reference's own code (both on the CPU).

Cells are spherocylinders of diameter 0.5; a cell of length L centred at c
with unit axis t has the segment c +- (L/2 - 0.25) t (getParticleEndpoints,
spatial/CollisionDetector.cpp:61-75), and a pair's separation is the segment
distance minus 0.5 (tryCreateConstraint, CollisionDetector.cpp:201-311).
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from helpers import normalized_contacts
from oracles import OracleColony, RefColony
from pcc_b200 import abi


def two_cells(c0, th0, c1, th1, L0=1.0, L1=1.0):
    q = lambda th: (math.cos(th / 2), math.sin(th / 2))  # noqa: E731  rotation about z
    return {"x": [c0[0], c1[0]], "y": [c0[1], c1[1]], "z": [0.0, 0.0],
            "q0": [q(th0)[0], q(th1)[0]], "q1": [0.0, 0.0], "q2": [0.0, 0.0], "q3": [q(th0)[1], q(th1)[1]],
            "length": [L0, L1], "l0": [1.0, 1.0], "diameter": [0.5, 0.5], "age": [1, 1]}


# (cells, expected separation, expected |normal| direction (up to sign), stress weights s_i, s_j)
CASES = {
    # side by side, parallel along x, centres 0.45 apart in y: segments 0.45 apart
    "parallel_side_by_side": (two_cells((0, 0), 0.0, (0, 0.45), 0.0), 0.45 - 0.5, (0, 1, 0), (0.0, 0.0)),
    # end to end along x: segments [-0.25, 0.25] and [0.7, 1.2], gap 0.45
    "end_to_end": (two_cells((0, 0), 0.0, (0.95, 0), 0.0), 0.45 - 0.5, (1, 0, 0), (0.5, 0.5)),
    # crossing at right angles: the segments intersect, distance 0, normal falls back to (1, 0, 0)
    "crossing": (two_cells((0, 0), 0.0, (0.1, 0.05), math.pi / 2), -0.5, (1, 0, 0), None),
    # tip to tip at a right angle: segment ends (0.25, 0) and (0.25 + 0.4, 0) ... second cell
    # vertical with its lower end 0.4 to the right of the first cell's right end
    "tip_to_tip": (two_cells((0, 0), 0.0, (0.65, 0.25), math.pi / 2), 0.4 - 0.5, (1, 0, 0), (0.5, 0.0)),
    # collinear and overlapping: distance 0 along the shared line
    "collinear_overlap": (two_cells((0, 0), 0.0, (0.3, 0), 0.0), -0.5, (1, 0, 0), None),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_contact_geometry_known_answers(name):
    cells, sd, ndir, weights = CASES[name]
    p = abi.default_params(ghost_mode=abi.GHOSTS_NONE)
    got = []
    for cls in (OracleColony, RefColony):
        col = cls(p)
        col.set_cells(cells)
        got.append(normalized_contacts(col.detect(0.25, 0)))
    o, r = got
    for k in o:  # the restatement is the reference, bit for bit
        np.testing.assert_array_equal(o[k], r[k], err_msg=k)
    assert o["gid_i"].tolist() == [0] and o["gid_j"].tolist() == [1]
    assert abs(o["sd"][0] - sd) < 1e-15
    n = o["normal"][0]
    assert abs(abs(float(np.dot(n, ndir))) - 1.0) < 1e-15
    if weights is not None:
        assert abs(o["stress_i"][0] - weights[0]) < 1e-15 and abs(o["stress_j"][0] - weights[1]) < 1e-15
    # contact point: midpoint of the closest points, r_i / r_j measured from the centres
    cp = o["contact_point"][0]
    np.testing.assert_allclose(o["r_i"][0], cp - np.array([cells["x"][0], cells["y"][0], 0.0]), atol=1e-15)
    np.testing.assert_allclose(o["r_j"][0], cp - np.array([cells["x"][1], cells["y"][1], 0.0]), atol=1e-15)


def test_separated_pair_is_not_a_contact():
    cells = two_cells((0, 0), 0.0, (0, 0.5 + 0.25 + 1e-6), 0.0)  # gap just beyond the 0.25 reach
    for cls in (OracleColony, RefColony):
        col = cls(abi.default_params(ghost_mode=abi.GHOSTS_NONE))
        col.set_cells(cells)
        assert col.detect(0.25, 0)["gid_i"].size == 0


def test_two_cell_lcp_closed_form():
    """Two cells end to end, overlapping by 0.01, growth switched off (tau huge):
    the LCP has one active row with A = D M D^T = 1/(xi l_i) + 1/(xi l_j) and
    phi_next(gamma) = Phi + dt A (gamma - gamma_0) = 0, so
    gamma* = gamma_0 - Phi / (dt A), and the solved pair just touches."""
    cells = two_cells((0, 0), 0.0, (0.99, 0), 0.0)
    dt, tol = 1e-3, 1e-9
    p = abi.default_params(dt=dt, fixed_dt=1, tau=1e12, tolerance=tol, ghost_mode=abi.GHOSTS_NONE)
    for cls in (OracleColony, RefColony):
        col = cls(p)
        col.set_cells(cells)
        st = col.solve(dt, 1)
        assert st["max_overlap"] <= tol and st["residual"] <= tol
        k = col.constraints()
        phase0 = k["phase"] == 0
        sd0 = -0.01
        a = 1.0 / 1.0 + 1.0 / 1.0
        gamma0 = 500.0 * 0.01
        want = gamma0 - sd0 / (dt * a)
        # the returned gamma is the previous iterate; it meets the closed form to the solver tolerance
        assert abs(k["gamma"][phase0][0] - want) / want < 1e-5
        after = col.get_cells()
        gap = (after["x"][1] - 0.25) - (after["x"][0] + 0.25) - 0.5
        assert abs(gap) < 1e-6
