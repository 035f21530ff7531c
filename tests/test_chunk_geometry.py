"""The BBPGD reduction chunks, checked on the CPU: tests/chunk_geometry.cu is
compiled by nvcc against the solver's own header and runs as host code (the
chunk functions are __host__ __device__), so no GPU is needed.  Every solver
form cuts the constraints with these functions, which is what keeps their
results bit-identical; the program checks the partition over constraint
counts from 0 to 5e7 for the targets in use."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.skipif(shutil.which("nvcc") is None and not Path("/usr/local/cuda/bin/nvcc").exists(),
                    reason="nvcc not found")
def test_chunks_partition_the_constraints(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = tmp_path / "chunk_geometry"
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17",
                    f"-I{ROOT / 'include'}", f"-I{ROOT / 'proliferatingcellcollectives-idp_b200' / 'csrc'}",
                    str(ROOT / "tests" / "chunk_geometry.cu"), "-o", str(exe)], check=True, timeout=300)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.startswith("ok"), r.stdout + r.stderr
