"""Host binding of the device library (libpcc_gpu.so) through its C ABI.

`Colony` is the Python face of one pcc_ctx: one colony resident on one GPU.
Its methods follow the reference's step interface -- `solve` is
ParticleManager::step (solveHardModel / solveSoftPotential), `step` is one
iteration of Domain::run -- and raise RuntimeError with the reference's
messages when the C ABI returns an error status.  There is no CPU fallback:
if the library is missing or no GPU is visible, construction fails.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

from . import abi

LIB_PATH = Path(__file__).resolve().parent / "libpcc_gpu.so"
_LIB = None


def load_library(path: str | os.PathLike | None = None):
    """Load libpcc_gpu.so (built by build.py).  Raises if it is missing."""
    global _LIB
    if _LIB is not None:
        return _LIB
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"{p} is missing: build the CUDA library first (python -c 'import __graft_entry__ as g; g.build()')")
    lib = C.CDLL(str(p))
    P = C.POINTER
    VP = C.c_void_p
    lib.pcc_default_params.argtypes = [P(abi.Params)]
    lib.pcc_create.argtypes = [P(abi.Params), C.c_int, P(VP)]
    lib.pcc_destroy.argtypes = [VP]
    lib.pcc_last_error.restype = C.c_char_p
    lib.pcc_last_error.argtypes = [VP]
    lib.pcc_set_dt.argtypes = [VP, C.c_double]
    lib.pcc_get_dt.argtypes = [VP, P(C.c_double)]
    lib.pcc_upload_cells.argtypes = [VP, P(abi.Cells), C.c_size_t]
    lib.pcc_download_cells.argtypes = [VP, P(abi.Cells), C.c_size_t, P(C.c_size_t)]
    lib.pcc_cell_count.argtypes = [VP, P(C.c_size_t)]
    lib.pcc_solve.argtypes = [VP, C.c_double, C.c_int, P(abi.StepStats)]
    lib.pcc_step.argtypes = [VP, P(abi.StepStats)]
    lib.pcc_run.argtypes = [VP, C.c_double, C.c_longlong, P(C.c_longlong), P(C.c_double), P(abi.StepStats)]
    lib.pcc_detect_contacts.argtypes = [VP, C.c_double, C.c_int, P(abi.Contacts), C.c_size_t, P(C.c_size_t)]
    lib.pcc_get_constraints.argtypes = [VP, P(abi.Contacts), C.c_size_t, P(C.c_size_t)]
    lib.pcc_bbpgd_frozen.argtypes = [VP, C.c_double, C.c_int, P(C.c_longlong), P(C.c_double), P(C.c_float)]
    lib.pcc_soft_forces_frozen.argtypes = [VP, C.c_int, P(C.c_float)]
    lib.pcc_set_profiling.argtypes = [VP, C.c_int]
    lib.pcc_reset_profile.argtypes = [VP]
    lib.pcc_get_profile.argtypes = [VP, P(abi.Profile)]
    lib.pcc_serve.argtypes = [P(abi.Job), C.c_size_t, C.c_int, C.c_double, C.c_int, P(abi.JobResult),
                              P(C.c_double)]
    lib.pcc_server_create.argtypes = [C.c_int, C.c_double, C.c_int, P(VP)]
    lib.pcc_server_submit.argtypes = [VP, P(abi.Job), P(C.c_ulonglong)]
    lib.pcc_server_poll.argtypes = [VP, P(abi.JobResult), P(C.c_ulonglong), C.c_size_t, P(C.c_size_t), C.c_double]
    lib.pcc_server_pending.argtypes = [VP, P(C.c_size_t), P(C.c_size_t)]
    lib.pcc_server_destroy.argtypes = [VP]
    lib.pcc_batch_create.argtypes = [P(abi.Params), C.c_int, C.c_int, P(VP)]
    lib.pcc_batch_context.argtypes = [VP, C.c_int, P(VP)]
    lib.pcc_batch_step.argtypes = [VP, P(abi.StepStats)]
    lib.pcc_batch_destroy.argtypes = [VP]
    lib.pcc_get_stream.restype = VP
    lib.pcc_get_stream.argtypes = [VP]
    lib.pcc_launch_count.restype = C.c_longlong
    lib.pcc_launch_count.argtypes = [VP]
    lib.pcc_division_seed.restype = C.c_uint
    lib.pcc_division_seed.argtypes = [C.c_ulonglong, C.c_ulonglong]
    lib.pcc_vtk_write_particles.argtypes = [C.c_char_p, C.c_char_p, C.c_ulonglong, P(abi.Cells), C.c_size_t, C.c_int]
    lib.pcc_vtk_write_simulation.argtypes = [C.c_char_p, C.c_ulonglong, P(abi.SimRecord)]
    lib.pcc_vtk_write_parameters.argtypes = [C.c_char_p, C.c_ulonglong, P(abi.Params)]
    lib.pcc_log_vtk.argtypes = [VP, C.c_char_p, C.c_ulonglong, P(abi.SimRecord)]
    lib.pcc_log_vtk_wait.argtypes = [VP]
    lib.pcc_vtk_load.argtypes = [C.c_char_p, P(abi.Cells), C.c_size_t, P(C.c_size_t), P(C.c_double),
                                 P(C.c_longlong), P(C.c_double)]
    lib.pcc_set_clock.argtypes = [VP, C.c_double, C.c_longlong]
    lib.pcc_set_trace_dir.argtypes = [VP, C.c_char_p]
    lib.pcc_get_bbpgd_trace.argtypes = [VP, P(abi.TraceStep), C.c_size_t, P(C.c_size_t)]
    lib.pcc_vtk_write_trace.argtypes = [C.c_char_p, C.c_ulonglong, P(abi.TraceStep), C.c_size_t]
    lib.pcc_division_length_host.restype = C.c_double
    lib.pcc_division_length_host.argtypes = [C.c_ulonglong, C.c_ulonglong, C.c_double]
    _LIB = lib
    return lib


# Messages the reference raises for the same conditions.
_REFERENCE_MESSAGES = {
    abi.PCC_ERR_NOCONV_BBPGD: "BBPGD did not converge",
    abi.PCC_ERR_NOCONV_RELCP: "Maximum number of constraint iterations reached",
}


class PccError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(msg)
        self.status = status


class Colony:
    """One colony resident on one GPU (a pcc_ctx)."""

    def __init__(self, params: abi.Params, device: int = 0):
        self.lib = load_library()
        self.h = C.c_void_p()
        rc = self.lib.pcc_create(C.byref(params), device, C.byref(self.h))
        if rc != 0:
            raise PccError(rc, f"pcc_create failed: {abi.STATUS_NAMES.get(rc, rc)}")
        self.n_cells_hint = 1024

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self.lib.pcc_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str):
        if rc != 0:
            msg = self.lib.pcc_last_error(self.h)
            msg = msg.decode() if msg else ""
            raise PccError(rc, _REFERENCE_MESSAGES.get(rc, f"{what}: {abi.STATUS_NAMES.get(rc, rc)}: {msg}"))

    # state transfer
    def set_cells(self, cells: dict):
        ca = abi.CellArrays.from_dict(cells)
        self._check(self.lib.pcc_upload_cells(self.h, C.byref(ca.struct), len(cells["x"])), "upload")

    def upload(self, ca: abi.CellArrays, n: int):
        self._check(self.lib.pcc_upload_cells(self.h, C.byref(ca.struct), n), "upload")

    def download(self, ca: abi.CellArrays) -> int:
        n = C.c_size_t(0)
        self._check(self.lib.pcc_download_cells(self.h, C.byref(ca.struct), ca.cap, C.byref(n)), "download")
        return int(n.value)

    @property
    def n_cells(self) -> int:
        n = C.c_size_t(0)
        self._check(self.lib.pcc_cell_count(self.h, C.byref(n)), "count")
        return int(n.value)

    def get_cells(self) -> dict:
        n = self.n_cells
        ca = abi.CellArrays(n)
        self.download(ca)
        return ca.to_dict(n)

    # solver / driver
    def solve(self, dt: float, it: int = 0) -> dict:
        st = abi.StepStats()
        self._check(self.lib.pcc_solve(self.h, dt, it, C.byref(st)), "solve")
        return st.as_dict()

    def step(self) -> dict:
        st = abi.StepStats()
        self._check(self.lib.pcc_step(self.h, C.byref(st)), "step")
        return st.as_dict()

    def run(self, end_radius: float, max_steps: int):
        steps = C.c_longlong(0)
        cs = C.c_double(0)
        st = abi.StepStats()
        self._check(self.lib.pcc_run(self.h, end_radius, max_steps, C.byref(steps), C.byref(cs), C.byref(st)), "run")
        return int(steps.value), float(cs.value), st.as_dict()

    def _contacts(self, fn, *args) -> dict:
        n = C.c_size_t(0)
        self._check(fn(self.h, *args, None, 0, C.byref(n)), "contacts")
        ca = abi.ContactArrays(int(n.value))
        self._check(fn(self.h, *args, C.byref(ca.struct), ca.cap, C.byref(n)), "contacts")
        return ca.to_dict(int(n.value))

    def detect(self, tol: float, phase: int = 0) -> dict:
        return self._contacts(self.lib.pcc_detect_contacts, C.c_double(tol), C.c_int(phase))

    def constraints(self) -> dict:
        return self._contacts(self.lib.pcc_get_constraints)

    def bbpgd_frozen(self, dt: float, repeats: int = 1):
        it = C.c_longlong(0)
        res = C.c_double(0)
        ms = C.c_float(0)
        self._check(self.lib.pcc_bbpgd_frozen(self.h, dt, repeats, C.byref(it), C.byref(res), C.byref(ms)), "bbpgd")
        return int(it.value), float(res.value), float(ms.value)

    def soft_forces_frozen(self, repeats: int = 1) -> float:
        ms = C.c_float(0)
        self._check(self.lib.pcc_soft_forces_frozen(self.h, repeats, C.byref(ms)), "soft")
        return float(ms.value)

    @property
    def dt(self) -> float:
        v = C.c_double(0)
        self._check(self.lib.pcc_get_dt(self.h, C.byref(v)), "dt")
        return v.value

    @dt.setter
    def dt(self, v: float):
        self._check(self.lib.pcc_set_dt(self.h, v), "dt")

    def profiling(self, on: bool = True):
        self._check(self.lib.pcc_set_profiling(self.h, 1 if on else 0), "profiling")
        self._check(self.lib.pcc_reset_profile(self.h), "profiling")

    def profile(self) -> dict:
        pr = abi.Profile()
        self._check(self.lib.pcc_get_profile(self.h, C.byref(pr)), "profile")
        return pr.as_dict()

    # VTK output / restart
    def log_vtk(self, outdir: str, index: int, record: dict | None = None):
        """Queue a log point (particles_, ghost_particles_ and, with a record,
        simulation_ files of `index`); returns before the files are written."""
        rec = sim_record(record) if record is not None else None
        self._check(self.lib.pcc_log_vtk(self.h, str(outdir).encode(), int(index),
                                         C.byref(rec) if rec is not None else None), "log_vtk")

    def log_vtk_wait(self):
        self._check(self.lib.pcc_log_vtk_wait(self.h), "log_vtk_wait")

    def set_trace_dir(self, path: str):
        self._check(self.lib.pcc_set_trace_dir(self.h, str(path).encode()), "set_trace_dir")

    def bbpgd_trace(self) -> list[dict]:
        """Records of the last traced hard-model solve (params.log_bbpgd_trace)."""
        n = C.c_size_t(0)
        self._check(self.lib.pcc_get_bbpgd_trace(self.h, None, 0, C.byref(n)), "trace")
        arr = (abi.TraceStep * max(int(n.value), 1))()
        self._check(self.lib.pcc_get_bbpgd_trace(self.h, arr, int(n.value), C.byref(n)), "trace")
        return [arr[i].as_dict() for i in range(int(n.value))]

    def set_clock(self, sim_time: float, iteration: int):
        self._check(self.lib.pcc_set_clock(self.h, float(sim_time), int(iteration)), "set_clock")

    @property
    def stream(self) -> int:
        return int(self.lib.pcc_get_stream(self.h) or 0)

    @property
    def launches(self) -> int:
        return int(self.lib.pcc_launch_count(self.h))


def serve(jobs: list[dict], slots: int, hbm_budget_bytes: float = 150e9, device: int = 0, check: bool = True):
    """Runs colony jobs with continuous batching (pcc_serve).  Each job is a
    dict with 'params' (abi.Params), 'end_radius' and optional 'arrival_s',
    'max_steps'.  Returns (list of result dicts, wall seconds); with check,
    raises PccError if a job failed (else each result carries its status)."""
    lib = load_library()
    n = len(jobs)
    arr = (abi.Job * max(n, 1))()
    for i, j in enumerate(jobs):
        arr[i].params = j["params"]
        arr[i].end_radius = float(j["end_radius"])
        arr[i].arrival_s = float(j.get("arrival_s", 0.0))
        arr[i].max_steps = int(j.get("max_steps", 0))
    res = (abi.JobResult * max(n, 1))()
    wall = C.c_double(0)
    rc = lib.pcc_serve(arr, n, int(slots), float(hbm_budget_bytes), device, res, C.byref(wall))
    out = [res[i].as_dict() for i in range(n)]
    if rc != 0 and (check or rc in (abi.PCC_ERR_INVALID, abi.PCC_ERR_CAPACITY)):
        raise PccError(rc, _REFERENCE_MESSAGES.get(rc, f"pcc_serve: {abi.STATUS_NAMES.get(rc, rc)}"))
    return out, wall.value


def division_length(seed: int, k: int, length: float) -> float:
    return load_library().pcc_division_length_host(seed, k, length)


def sim_record(d: dict) -> abi.SimRecord:
    r = abi.SimRecord()
    for k, v in d.items():
        setattr(r, k, v)
    return r


def write_particles(outdir: str, prefix: str, index: int, cells: dict, ghost_copies: bool = False):
    """Host-only writer of a particle file pair in the reference's format."""
    n = len(cells["x"])
    ca = abi.CellArrays.from_dict(cells)
    rc = load_library().pcc_vtk_write_particles(str(outdir).encode(), prefix.encode(), int(index),
                                                C.byref(ca.struct), n, 1 if ghost_copies else 0)
    if rc != 0:
        raise PccError(rc, "pcc_vtk_write_particles failed")


def write_simulation(outdir: str, index: int, record: dict):
    rc = load_library().pcc_vtk_write_simulation(str(outdir).encode(), int(index), C.byref(sim_record(record)))
    if rc != 0:
        raise PccError(rc, "pcc_vtk_write_simulation failed")


def write_parameters(outdir: str, index: int, params: abi.Params):
    rc = load_library().pcc_vtk_write_parameters(str(outdir).encode(), int(index), C.byref(params))
    if rc != 0:
        raise PccError(rc, "pcc_vtk_write_parameters failed")


def load_vtk(path: str):
    """Restart state from a VTK output directory (or a file in it):
    (cells dict, simulation time, step, dt) as pcc_vtk_load returns them."""
    lib = load_library()
    n = C.c_size_t(0)
    t, dt = C.c_double(0), C.c_double(0)
    step = C.c_longlong(0)
    rc = lib.pcc_vtk_load(str(path).encode(), None, 0, C.byref(n), C.byref(t), C.byref(step), C.byref(dt))
    if rc != 0:
        raise PccError(rc, f"pcc_vtk_load: cannot read a VTK state from {path}")
    ca = abi.CellArrays(int(n.value))
    rc = lib.pcc_vtk_load(str(path).encode(), C.byref(ca.struct), ca.cap, C.byref(n), C.byref(t), C.byref(step),
                          C.byref(dt))
    if rc != 0:
        raise PccError(rc, f"pcc_vtk_load: cannot read a VTK state from {path}")
    return ca.to_dict(int(n.value)), t.value, int(step.value), dt.value


def write_trace(outdir: str, first_index: int, steps: list[dict]):
    """Host-only writer of bbpgdtrace files in the reference's format."""
    arr = (abi.TraceStep * max(len(steps), 1))()
    for i, d in enumerate(steps):
        for k, v in d.items():
            setattr(arr[i], k, v)
    rc = load_library().pcc_vtk_write_trace(str(outdir).encode(), int(first_index), arr, len(steps))
    if rc != 0:
        raise PccError(rc, "pcc_vtk_write_trace failed")


class Server:
    """A running request loop (pcc_server): submit colony jobs while it runs,
    poll finished results by id."""

    def __init__(self, slots: int, hbm_budget_bytes: float = 150e9, device: int = 0):
        self.lib = load_library()
        self.h = C.c_void_p()
        rc = self.lib.pcc_server_create(int(slots), float(hbm_budget_bytes), device, C.byref(self.h))
        if rc != 0:
            raise PccError(rc, "pcc_server_create failed")

    def submit(self, job: dict) -> int:
        j = abi.Job()
        j.params = job["params"]
        j.end_radius = float(job["end_radius"])
        j.arrival_s = 0.0
        j.max_steps = int(job.get("max_steps", 0))
        k = C.c_ulonglong(0)
        rc = self.lib.pcc_server_submit(self.h, C.byref(j), C.byref(k))
        if rc != 0:
            raise PccError(rc, f"pcc_server_submit: {abi.STATUS_NAMES.get(rc, rc)}")
        return int(k.value)

    def poll(self, wait_s: float = 0.0, cap: int = 64) -> dict:
        res = (abi.JobResult * cap)()
        ids = (C.c_ulonglong * cap)()
        n = C.c_size_t(0)
        rc = self.lib.pcc_server_poll(self.h, res, ids, cap, C.byref(n), float(wait_s))
        if rc != 0:
            raise PccError(rc, "pcc_server_poll failed")
        return {int(ids[i]): res[i].as_dict() for i in range(int(n.value))}

    def pending(self) -> tuple[int, int]:
        q, r = C.c_size_t(0), C.c_size_t(0)
        self.lib.pcc_server_pending(self.h, C.byref(q), C.byref(r))
        return int(q.value), int(r.value)

    def close(self):
        if self.h:
            self.lib.pcc_server_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _BorrowedColony(Colony):
    """A colony whose context belongs to a Batch (not destroyed here)."""

    def __init__(self, lib, handle):  # noqa: D107 - no pcc_create
        self.lib = lib
        self.h = handle

    def close(self):
        self.h = C.c_void_p()


class Batch:
    """Colonies stepped together (pcc_batch): batch.step() advances every
    colony once; batch[k] is colony k (upload, download, queries)."""

    def __init__(self, params: list, device: int = 0):
        self.lib = load_library()
        arr = (abi.Params * len(params))(*params)
        self.h = C.c_void_p()
        rc = self.lib.pcc_batch_create(arr, len(params), device, C.byref(self.h))
        if rc != 0:
            raise PccError(rc, "pcc_batch_create failed")
        self.n = len(params)
        self._cols = []
        for k in range(self.n):
            c = C.c_void_p()
            self.lib.pcc_batch_context(self.h, k, C.byref(c))
            self._cols.append(_BorrowedColony(self.lib, c))

    def __getitem__(self, k: int) -> Colony:
        return self._cols[k]

    def step(self) -> list[dict]:
        st = (abi.StepStats * self.n)()
        rc = self.lib.pcc_batch_step(self.h, st)
        if rc != 0:
            raise PccError(rc, _REFERENCE_MESSAGES.get(rc, f"pcc_batch_step: {abi.STATUS_NAMES.get(rc, rc)}"))
        return [st[k].as_dict() for k in range(self.n)]

    def close(self):
        if self.h:
            for c in self._cols:
                c.close()
            self.lib.pcc_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
