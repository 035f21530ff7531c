"""VTK log points of a device colony: the asynchronous snapshot writer
(pcc_log_vtk) against the host writer on the same state, and a restart from
the written files."""
from __future__ import annotations

import filecmp

import numpy as np
import pytest

from helpers import load_fixture, params_of, sub
from pcc_b200 import device
from pcc_b200.device import Colony

pytestmark = pytest.mark.gpu

RECORD = dict(simulation_time_s=0.5, time_since_last_log_s=0.25, step=7, num_particles=256, num_constraints=2654,
              colony_radius=10.5, recursive_iterations=4, bbpgd_iterations=130, max_overlap=3.5e-4,
              residual=1e-4, dt_s=0.001, memory_usage_mb=1.0, peak_memory_mb=2.0, cpu_time_s=3.0,
              mpi_comm_time_s=4.0, load_imbalance=1.0)


def test_async_log_matches_host_writer(tmp_path):
    fx = load_fixture("hard_r10_seed3")
    p = params_of(fx)
    g = Colony(p)
    g.set_cells(sub(fx, "cells_"))
    g.solve(p.dt, 0)
    states = []
    for k in range(2):
        states.append(g.get_cells())
        g.log_vtk(str(tmp_path / "dev"), k, RECORD)
        g.step()  # the colony steps on while the snapshot is written
    g.log_vtk_wait()
    for k, cells in enumerate(states):
        device.write_particles(str(tmp_path / "host"), "particles", k, cells)
        device.write_particles(str(tmp_path / "host"), "ghost_particles", k, cells, ghost_copies=True)
        device.write_simulation(str(tmp_path / "host"), k, RECORD)
        for pre in ("particles", "ghost_particles", "simulation"):
            base = f"{pre}_{k:07d}"
            assert filecmp.cmp(tmp_path / "dev" / f"{base}.pvtu", tmp_path / "host" / f"{base}.pvtu", shallow=False)
            assert filecmp.cmp(tmp_path / "dev" / "data" / f"{base}_rank_0000.vtu",
                               tmp_path / "host" / "data" / f"{base}_rank_0000.vtu", shallow=False), base


def test_restart_from_logged_state(tmp_path):
    fx = load_fixture("hard_r10_seed3")
    p = params_of(fx)
    g = Colony(p)
    g.set_cells(sub(fx, "cells_"))
    g.step()
    before = g.get_cells()
    g.log_vtk(str(tmp_path), 0, RECORD)
    g.log_vtk_wait()
    cells, t, step, dt = device.load_vtk(str(tmp_path))
    assert (t, step) == (0.5, 7)
    assert np.max(np.abs(cells["x"] - before["x"])) < 1e-4
    h = Colony(p)
    h.set_cells(cells)
    h.set_clock(t, step)
    st = h.step()
    assert st["n_cells"] >= len(cells["x"]) and st["max_overlap"] <= p.tolerance


def test_bbpgd_trace_matches_reference(tmp_path):
    """-log_bbgd_trace: residual tested every iteration and one record per
    iteration with the energy terms; the device records follow the
    reference's within rounding of the (reordered) sums."""
    from oracles import RefColony
    from test_vtk import read_trace_dir
    fx = load_fixture("hard_r10_seed3")
    p = params_of(fx, log_bbpgd_trace=1)
    ref = RefColony(p, outdir=str(tmp_path / "ref"))
    ref.set_cells(sub(fx, "cells_"))
    sr = ref.solve(p.dt, 0)
    want = read_trace_dir(tmp_path / "ref" / "logs")
    g = Colony(p)
    g.set_trace_dir(str(tmp_path / "dev"))
    g.set_cells(sub(fx, "cells_"))
    sg = g.solve(p.dt, 0)
    got = g.bbpgd_trace()
    assert sg["relcp_iterations"] == sr["relcp_iterations"]
    assert [r["step"] for r in got] == [r["step"] for r in want]
    assert [r["recursive_iteration"] for r in got] == [r["recursive_iteration"] for r in want]
    assert [r["total_constraints"] for r in got] == [r["total_constraints"] for r in want]
    for k in ("residual", "step_size", "linear", "quadratic", "growth", "total"):
        a = np.array([r[k] for r in got])
        b = np.array([r[k] for r in want])  # 6 significant digits in the files
        np.testing.assert_allclose(a, b, rtol=2e-5, atol=1e-12, err_msg=k)
    # the same records are on disk in the trace directory
    assert len(read_trace_dir(tmp_path / "dev")) == len(got)
    # a step that is not a multiple of 10 is not traced
    g2 = Colony(p)
    g2.set_cells(sub(fx, "cells_"))
    g2.solve(p.dt, 3)
    assert g2.bbpgd_trace() == []


def test_command_line_driver_logs_and_restarts(tmp_path):
    """The C++ driver with the reference's options writes the reference's
    output tree and restarts from it with -starter_vtk."""
    import subprocess
    from pathlib import Path
    exe = Path(__file__).resolve().parents[1] / "proliferatingcellcollectives-idp_b200" / "pcc_cellcollectives"
    run = subprocess.run([str(exe), "-mode", "hard", "-dt", "1e-3", "-fixed_dt", "1", "-end_radius", "2.5",
                          "-seed", "3"], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert run.returncode == 0, run.stderr
    out = tmp_path / "vtk_output_hard"
    assert (out / "parameters_0000000.pvtu").exists()
    logs = sorted(out.glob("particles_*.pvtu"))
    sims = sorted(out.glob("simulation_*.pvtu"))
    assert len(logs) >= 3 and len(logs) == len(sims)
    assert len(sorted((out / "data").glob("ghost_particles_*_rank_0000.vtu"))) == len(logs)
    cells, t, step, dt = device.load_vtk(str(out))
    assert len(cells["x"]) >= 2 and t > 0 and step > 0
    again = subprocess.run([str(exe), "-mode", "hard", "-dt", "1e-3", "-fixed_dt", "1", "-end_radius", "3.0",
                            "-starter_vtk", str(out)], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert again.returncode == 0, again.stderr
    assert f"Loading {len(cells['x'])} particles" in again.stdout
    assert len(sorted(out.glob("particles_*.pvtu"))) > len(logs)
