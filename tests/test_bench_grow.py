"""bench.py --grow on the CPU with a stand-in colony: a run split into
pieces by --checkpoint / --resume reports the same totals as the same run in
one piece, each resumed piece starts from the saved state and clock, and
draws its division lengths from its own stream (seed + piece index).  The
device colony is replaced by a counter that grows by one cell and one length
unit of radius per step, so only the bookkeeping is under test."""
from __future__ import annotations

import io
import json
import sys
from contextlib import redirect_stdout
from pathlib import Path
from types import SimpleNamespace

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


class _Event:
    def __init__(self, **kw):
        self.t = 0.0

    def record(self, stream=None):
        import time
        self.t = time.time()

    def synchronize(self):
        pass

    def elapsed_time(self, other):
        return (other.t - self.t) * 1e3


class _Colony:
    """Grows one cell and one unit of radius per step."""

    made: list = []
    stream = 0

    def __init__(self, params):
        self.n, self.r, self._dt, self.t, self.seed = 1, 0.0, params.dt, 0.0, int(params.seed)
        self.clock = None
        _Colony.made.append(self)

    def set_cells(self, c):
        self.n = len(c["x"])
        self.r = float(np.max(np.abs(c["x"]))) if self.n > 1 else 0.0

    @property
    def dt(self):
        return self._dt

    @dt.setter
    def dt(self, v):
        self._dt = v

    def set_clock(self, t, it):
        self.t, self.clock = t, (t, it)

    def profiling(self, on):
        pass

    def profile(self):
        return {"bbpgd_ms": 1.0, "detect_ms": 2.0, "solve_ms": 3.0}

    def step(self):
        self.n += 1
        self.r += 1.0
        self.t += self._dt
        return {"n_cells": self.n, "bbpgd_iterations": 10, "colony_radius": self.r, "dt_used": self._dt,
                "sim_time": self.t, "relcp_iterations": 2}

    def get_cells(self):
        n = self.n
        d = {"x": np.arange(n, dtype=float) * (self.r / max(n - 1, 1))}
        for k in ("y", "z", "q1", "q2", "q3", "ldot", "impedance", "stress"):
            d[k] = np.zeros(n)
        d["q0"], d["length"], d["l0"], d["diameter"] = np.ones(n), np.ones(n), np.ones(n), np.full(n, 0.5)
        d["age"], d["num_constraints"] = np.zeros(n, np.int32), np.zeros(n, np.int32)
        d["force"], d["velocity"] = np.zeros((n, 6)), np.zeros((n, 6))
        return d


@pytest.fixture
def grow(monkeypatch):
    import torch

    import bench
    from pcc_b200 import build, device
    monkeypatch.setattr(build, "build", lambda *a, **k: None)
    monkeypatch.setattr(device, "Colony", _Colony)
    monkeypatch.setattr(torch.cuda, "init", lambda: None)
    monkeypatch.setattr(torch.cuda, "Event", _Event)
    monkeypatch.setattr(torch.cuda, "ExternalStream", lambda *a, **k: None)
    monkeypatch.setattr(bench, "packing_fraction", lambda cells: 0.5)
    _Colony.made = []

    def run(max_steps: int, **kw):
        a = SimpleNamespace(precision="mixed", radius=30.0, job_seed=0, grow_seconds=1e9, save="", checkpoint="",
                            resume="")
        for k, v in kw.items():
            setattr(a, k, v)
        real = _Colony.step
        count = {"n": 0}

        def limited(self):
            count["n"] += 1
            if count["n"] >= max_steps:
                a.grow_seconds = -1.0  # the time limit ends the piece after this step
            return real(self)

        monkeypatch.setattr(_Colony, "step", limited)
        out = io.StringIO()
        with redirect_stdout(out):
            bench.run_grow(a)
        monkeypatch.setattr(_Colony, "step", real)
        return json.loads(out.getvalue().strip().splitlines()[-1])

    return run


def test_resumed_pieces_add_up_to_one_run(grow, tmp_path):
    whole = grow(10**9)
    ck = str(tmp_path / "ck.npz")
    first = grow(12, checkpoint=ck)
    second = grow(12, resume=ck, checkpoint=ck)
    last = grow(10**9, resume=ck, checkpoint=ck, save=str(tmp_path / "snap.npz"))
    assert whole["reached"] and last["reached"] and not first["reached"] and not second["reached"]
    assert [first["segments"], second["segments"], last["segments"]] == [1, 2, 3]
    for k in ("steps", "cell_steps", "bbpgd_iterations", "radius"):
        assert last[k] == whole[k], k
    assert last["stage_ms"] == {"bbpgd": 3.0, "detect": 6.0, "solve": 9.0}
    assert [m["step"] for m in last["marks"]] == [m["step"] for m in whole["marks"]]
    # each piece draws from its own division stream and starts from the saved clock
    assert [c.seed for c in _Colony.made] == [0, 0, 1, 2]
    assert _Colony.made[2].clock == (pytest.approx(12e-3), 12)
    assert _Colony.made[3].clock == (pytest.approx(24e-3), 24)
    saved = np.load(ck)
    assert "cell_force" not in saved.files and "cell_velocity" not in saved.files
    assert saved["cell_x"].dtype == np.float64 and saved["cell_x"].size == last["cells"]
    snap = np.load(tmp_path / "snap.npz")
    assert int(snap["steps"]) == whole["steps"] and snap["x"].dtype == np.float32
