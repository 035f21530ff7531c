"""The command-line driver's option handling, which runs before any device
work (no GPU needed): -help lists the reference's options with their
defaults, and a missing -mode fails with the reference's message."""
from __future__ import annotations

import subprocess
from pathlib import Path

EXE = Path(__file__).resolve().parents[1] / "proliferatingcellcollectives-idp_b200" / "pcc_cellcollectives"


def test_help_lists_reference_options():
    r = subprocess.run([str(EXE), "-help"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0
    for opt in ("-mode", "-dt", "-end_radius", "-log_every_colony_radius_delta", "-log_every_sim_time_delta",
                "-cfl_factor", "-log_bbgd_trace", "-starter_vtk", "-xi", "-tau", "-l0", "-lambda", "-kcc",
                "-tolerance", "-max_bbpgd_iterations", "-max_recursive_iterations", "-linked_cell_size"):
        assert opt in r.stdout, opt
    # defaults of util/CLIParser.h:165-195
    assert "[default: 0.01]" in r.stdout and "[default: 0.5]" in r.stdout and "[default: 20000]" in r.stdout


def test_missing_mode_is_an_error():
    r = subprocess.run([str(EXE), "-dt", "1e-3"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1
    assert "Error: Required parameter -mode not provided. Use -help for usage information." in r.stdout
