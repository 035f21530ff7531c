"""The multi-GPU form of the benchmark is N independent colony replicas, one
per rank, with no collective on the data path; only the timing is combined
(max over ranks) and the cell-steps are summed.  These tests run that host
logic with world size 2 on the gloo backend (CPU)."""
from __future__ import annotations

import os
import sys
from pathlib import Path

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _worker(rank: int, world: int, port: int, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    import pcc_pkg

    pcc_pkg.load_package()
    from pcc_b200 import abi
    from oracles import OracleColony

    import bench

    # each rank grows its own colony replica (different seed) on the CPU oracle
    p = abi.default_params(dt=1e-3, fixed_dt=1, seed=rank)
    o = OracleColony(p)
    o.set_cells(abi.seed_cell(rank))
    cells = sum(o.step()["n_cells"] for _ in range(800))
    ms = 100.0 + 50.0 * rank  # stand-in device times
    t = torch.tensor([ms], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor([float(cells)], dtype=torch.float64)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    gathered = [None] * world
    dist.all_gather_object(gathered, (float(cells), ms))
    value, tmax = bench.aggregate([g[0] for g in gathered], [g[1] for g in gathered])
    q.put((rank, float(t.item()), float(c.item()), value, tmax, cells))
    dist.destroy_process_group()


def test_replicas_aggregate_over_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 2000)
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    out = [q.get(timeout=240) for _ in procs]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    out.sort()
    (_, t0, c0, v0, m0, cells0), (_, t1, c1, v1, m1, cells1) = out
    assert t0 == t1 == 150.0                      # max over ranks
    assert c0 == c1 == cells0 + cells1            # cell-steps summed
    assert v0 == pytest.approx((cells0 + cells1) / 0.150)
    assert m0 == m1 == 150.0
    assert cells0 > 800 and cells1 > 800          # both replicas divided


def test_bench_starts_its_own_ranks():
    """`bench.py --gpus 2` without a launcher starts two ranks itself (the
    rendezvous on 127.0.0.1), and rank 0 reports the whole-job figure: the
    cell-steps of both replicas over the slowest rank's time (gloo here, NCCL
    on GPUs)."""
    import json
    import subprocess

    env = dict(os.environ, PCC_BENCH_BACKEND="gloo")
    env.pop("WORLD_SIZE", None)
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--gpus", "2", "--steps", "700",
                        "--replica-selftest"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(ln) for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    out = lines[0]
    assert out["n_gpus"] == 2
    assert out["ms_max"] == 150.0
    assert out["cell_steps"] > out["rank0_cell_steps"] >= 700
    assert out["value"] == pytest.approx(out["cell_steps"] / 0.150)
