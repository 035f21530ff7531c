"""VTK output and restart against the reference's own loggers and loader.

The reference's ParticleLogger / SimulationLogger / ParameterLogger and its
VTKStateLoader run from the compiled reference (oracle/_ref); the library's
host-side writers must produce the same bytes for the same cells and record,
and its loader must rebuild the same cells from the same files.
"""
from __future__ import annotations

import filecmp
from pathlib import Path

import numpy as np
import pytest

from helpers import load_fixture, params_of, sub
from oracles import RefColony, ref_load_vtk
from pcc_b200 import abi, device

RECORD = dict(simulation_time_s=1.2345678, time_since_last_log_s=3e-05, step=123, num_particles=256,
              num_constraints=2654, colony_radius=10.5, recursive_iterations=4, bbpgd_iterations=130,
              max_overlap=0.00035335, residual=1e-7, dt_s=0.001, memory_usage_mb=1234.5, peak_memory_mb=2e6,
              cpu_time_s=0.0, mpi_comm_time_s=12.0, load_imbalance=1.0)


def _same(a: Path, b: Path):
    assert a.exists() and b.exists(), (a, b)
    if not filecmp.cmp(a, b, shallow=False):
        la, lb = a.read_text().splitlines(), b.read_text().splitlines()
        for i, (x, y) in enumerate(zip(la, lb)):
            assert x == y, f"{a.name} line {i + 1}: {x[:200]!r} != {y[:200]!r}"
        assert len(la) == len(lb), (a.name, len(la), len(lb))


@pytest.fixture(scope="module")
def ref_logged(tmp_path_factory):
    fx = load_fixture("hard_r10_seed3")
    p = params_of(fx)
    ref = RefColony(p, outdir=str(tmp_path_factory.mktemp("ref")))
    ref.set_cells(sub(fx, "cells_"))
    ref.solve(p.dt, 0)
    ref.log_vtk(device.sim_record(RECORD))
    return p, ref, ref.get_cells()


def test_particle_file_byte_identical(ref_logged, tmp_path):
    p, ref, cells = ref_logged
    device.write_particles(str(tmp_path), "particles", 0, cells)
    _same(tmp_path / "particles_0000000.pvtu", ref.vtk_dir / "particles_0000000.pvtu")
    _same(tmp_path / "data" / "particles_0000000_rank_0000.vtu",
          ref.vtk_dir / "data" / "particles_0000000_rank_0000.vtu")


def test_simulation_file_byte_identical(ref_logged, tmp_path):
    p, ref, cells = ref_logged
    device.write_simulation(str(tmp_path), 0, RECORD)
    _same(tmp_path / "simulation_0000000.pvtu", ref.vtk_dir / "simulation_0000000.pvtu")
    _same(tmp_path / "data" / "simulation_0000000_rank_0000.vtu",
          ref.vtk_dir / "data" / "simulation_0000000_rank_0000.vtu")


def test_parameter_file_byte_identical(ref_logged, tmp_path):
    p, ref, cells = ref_logged
    q = abi.Params.from_buffer_copy(p)
    # the oracle driver builds its Domain with both log cadences at 0
    q.log_every_colony_radius_delta = 0.0
    q.log_every_sim_time_delta = 0.0
    device.write_parameters(str(tmp_path), 0, q)
    _same(tmp_path / "parameters_0000000.pvtu", ref.vtk_dir / "parameters_0000000.pvtu")
    _same(tmp_path / "data" / "parameters_0000000_rank_0000.vtu",
          ref.vtk_dir / "data" / "parameters_0000000_rank_0000.vtu")


def test_restart_loader_matches_reference_loader(ref_logged):
    p, ref, cells = ref_logged
    got, t, step, dt = device.load_vtk(str(ref.vtk_dir))
    want, t_ref, step_ref, dt_ref = ref_load_vtk(str(ref.vtk_dir))
    assert (t, step, dt) == (t_ref, step_ref, dt_ref)
    # the reference loader reads a field as the first run of digits, '.' and
    # '-' on its line: 3e-05 comes back as 3
    assert step == 123 and dt == 0.001 and t == 1.23457
    assert len(got["x"]) == len(want["x"]) == len(cells["x"])
    for k in ("x", "y", "z", "q0", "q1", "q2", "q3", "length", "l0", "diameter", "age", "force", "velocity"):
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)
    # positions come back at the file's float / 6-digit precision
    assert np.max(np.abs(got["x"] - cells["x"])) < 1e-4


def test_load_accepts_a_file_path_and_rejects_missing(ref_logged, tmp_path):
    p, ref, cells = ref_logged
    a = device.load_vtk(str(ref.vtk_dir / "particles_0000000.pvtu"))
    assert len(a[0]["x"]) == len(cells["x"])
    with pytest.raises(device.PccError):
        device.load_vtk(str(tmp_path / "nothing_here"))


def test_empty_colony_and_ghost_copies_write(tmp_path, ref_logged):
    p, ref, cells = ref_logged
    device.write_particles(str(tmp_path), "particles", 7, {k: v[:0] for k, v in cells.items()})
    text = (tmp_path / "data" / "particles_0000007_rank_0000.vtu").read_text()
    assert 'NumberOfPoints="0"' in text
    device.write_particles(str(tmp_path), "ghost_particles", 0, cells, ghost_copies=True)
    g = (tmp_path / "data" / "ghost_particles_0000000_rank_0000.vtu").read_text()
    r = np.hypot(cells["x"], cells["y"])
    ang = np.degrees(np.arctan2(cells["y"], cells["x"])) % 360.0
    # distance to the angle-0 boundary of the one sector: r sin(min(a, 360 - a)),
    # which is small near both ends of the x axis
    near = (r >= 8.0) & (r * np.sin(np.radians(np.minimum(ang, 360 - ang))) < 2.5)
    assert f'NumberOfPoints="{int(near.sum())}"' in g


def read_trace_dir(d: Path) -> list[dict]:
    """The records of bbpgdtrace_<k> files (k = 1, 2, ...) from their field data."""
    out = []
    k = 1
    while (d / f"bbpgdtrace_{k:07d}.pvtu").exists():
        text = (d / "data" / f"bbpgdtrace_{k:07d}_rank_0000.vtu").read_text().splitlines()
        rec = {}
        for i, line in enumerate(text):
            if "<DataArray" in line and "NumberOfTuples" in line:
                name = line.split('Name="')[1].split('"')[0]
                v = text[i + 1].strip()
                rec[name] = int(v) if name in ("step", "recursive_iteration", "total_constraints") else float(v)
        out.append(rec)
        k += 1
    return out


@pytest.fixture(scope="module")
def ref_trace(tmp_path_factory):
    fx = load_fixture("hard_r10_seed3")
    p = params_of(fx, log_bbpgd_trace=1)
    ref = RefColony(p, outdir=str(tmp_path_factory.mktemp("reftrace")))
    ref.set_cells(sub(fx, "cells_"))
    st = ref.solve(p.dt, 0)
    return p, Path(ref._tmp) / "logs", st


def test_trace_files_byte_identical(ref_trace, tmp_path):
    p, d, st = ref_trace
    recs = read_trace_dir(d)
    # one record per BBPGD iteration of every phase, residual tested every iteration
    assert len(recs) == sum(1 for r in recs if r["step"] == 0) + st["bbpgd_iterations"]
    device.write_trace(str(tmp_path), 1, recs)
    for k in (1, len(recs) // 2, len(recs)):
        _same(tmp_path / f"bbpgdtrace_{k:07d}.pvtu", d / f"bbpgdtrace_{k:07d}.pvtu")
        _same(tmp_path / "data" / f"bbpgdtrace_{k:07d}_rank_0000.vtu", d / "data" / f"bbpgdtrace_{k:07d}_rank_0000.vtu")


def test_restart_reads_field_values_as_the_reference_does(tmp_path, ref_logged):
    """VTKStateLoader reads a field value as the first run of digits, '.' and
    '-' on its line, so an exponent is dropped ("3e-05" -> 3); the restart
    loader keeps that reading."""
    p, ref, cells = ref_logged
    rec = dict(RECORD, dt_s=3e-05, simulation_time_s=2.5e-06, step=7)
    device.write_particles(str(tmp_path), "particles", 7, cells)
    device.write_simulation(str(tmp_path), 7, rec)
    got = device.load_vtk(str(tmp_path))
    want = ref_load_vtk(str(tmp_path))
    assert got[1:] == want[1:] == (2.5, 7, 3.0)
    for k in ("x", "y", "q0", "q3", "length", "force", "velocity"):
        np.testing.assert_array_equal(got[0][k], want[0][k], err_msg=k)
