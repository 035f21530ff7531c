import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(Path(__file__).resolve().parent))

import pcc_pkg  # noqa: E402

pcc_pkg.load_package()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA library)")
    config.addinivalue_line("markers", "slow: longer CPU oracle runs")


def pytest_sessionstart(session):
    """Bring the in-tree device library and the C oracle up to date (nvcc and
    gcc are both present wherever the tests run)."""
    import subprocess

    from pcc_b200 import build

    build.build()
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "oracle"], check=True)
