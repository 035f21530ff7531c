"""ctypes handles on the CPU oracles (test infrastructure only).

RefColony    -- the reference simulator's own C++ sources compiled in place
                against single-rank PETSc/MPI stand-ins (oracle/_ref/libpccref_*.so).
OracleColony -- the plain-C restatement in oracle/pcc_oracle.c
                (oracle/_ref/libpcc_oracle.so).
Both expose the same methods as the device handle in the package, so a
parity test drives all three the same way.
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile
from pathlib import Path

import numpy as np

from pcc_b200 import abi

REPO = Path(__file__).resolve().parents[1]
REF_DIR = REPO / "oracle" / "_ref"


def _load(name: str):
    path = REF_DIR / name
    if not path.exists():
        raise FileNotFoundError(f"{path} is missing: run `make -C oracle` (or __graft_entry__.build())")
    return C.CDLL(str(path))


_VP = C.c_void_p
_P = C.POINTER


def _bind_common(lib, prefix: str):
    f = lambda n: getattr(lib, prefix + n)  # noqa: E731
    f("create").restype = _VP
    f("create").argtypes = [_P(abi.Params), C.c_char_p] if prefix == "pcc_ref_" else [_P(abi.Params)]
    f("destroy").argtypes = [_VP]
    f("last_error").restype = C.c_char_p
    f("last_error").argtypes = [_VP]
    f("set_cells").argtypes = [_VP, _P(abi.Cells), C.c_size_t]
    f("get_cells").argtypes = [_VP, _P(abi.Cells), C.c_size_t, _P(C.c_size_t)]
    f("solve").argtypes = [_VP, C.c_double, C.c_int, _P(abi.StepStats)]
    f("step").argtypes = [_VP, _P(abi.StepStats)]
    f("run").argtypes = [_VP, C.c_double, C.c_longlong, _P(C.c_longlong), _P(C.c_double), _P(abi.StepStats)]
    f("detect").argtypes = [_VP, C.c_double, C.c_int, _P(abi.Contacts), C.c_size_t, _P(C.c_size_t)]
    f("get_constraints").argtypes = [_VP, _P(abi.Contacts), C.c_size_t, _P(C.c_size_t)]
    f("get_dt").restype = C.c_double
    f("get_dt").argtypes = [_VP]
    f("set_dt").argtypes = [_VP, C.c_double]
    f("colony_radius").restype = C.c_double
    f("colony_radius").argtypes = [_VP]
    f("division_count").restype = C.c_ulonglong
    f("division_count").argtypes = [_VP]


class _CpuColony:
    prefix = ""
    lib = None

    def _f(self, name):
        return getattr(self.lib, self.prefix + name)

    def _check(self, rc: int, what: str):
        if rc != 0:
            msg = self._f("last_error")(self.h)
            raise RuntimeError(f"{what}: {abi.STATUS_NAMES.get(rc, rc)}: {msg.decode() if msg else ''}")

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self._f("destroy")(h)
            self.h = None

    def set_cells(self, cells: dict):
        ca = abi.CellArrays.from_dict(cells)
        self._check(self._f("set_cells")(self.h, C.byref(ca.struct), len(cells["x"])), "set_cells")

    def get_cells(self) -> dict:
        n = C.c_size_t(0)
        rc = self._f("get_cells")(self.h, None, 0, C.byref(n)) if False else None
        cap = max(self.n_cells_hint, 1)
        while True:
            ca = abi.CellArrays(cap)
            rc = self._f("get_cells")(self.h, C.byref(ca.struct), cap, C.byref(n))
            if rc == abi.PCC_ERR_CAPACITY:
                cap = int(n.value)
                continue
            self._check(rc, "get_cells")
            self.n_cells_hint = int(n.value)
            return ca.to_dict(int(n.value))

    def solve(self, dt: float, it: int = 0) -> dict:
        st = abi.StepStats()
        self._check(self._f("solve")(self.h, dt, it, C.byref(st)), "solve")
        return st.as_dict()

    def step(self) -> dict:
        st = abi.StepStats()
        self._check(self._f("step")(self.h, C.byref(st)), "step")
        self.n_cells_hint = max(self.n_cells_hint, int(st.n_cells) * 2)
        return st.as_dict()

    def run(self, end_radius: float, max_steps: int):
        steps = C.c_longlong(0)
        cs = C.c_double(0)
        st = abi.StepStats()
        self._check(self._f("run")(self.h, end_radius, max_steps, C.byref(steps), C.byref(cs), C.byref(st)), "run")
        self.n_cells_hint = max(self.n_cells_hint, int(st.n_cells) * 2)
        return int(steps.value), float(cs.value), st.as_dict()

    def _contacts(self, fn, *args) -> dict:
        n = C.c_size_t(0)
        cap = 1024
        while True:
            ca = abi.ContactArrays(cap)
            rc = fn(self.h, *args, C.byref(ca.struct), cap, C.byref(n))
            if rc == abi.PCC_ERR_CAPACITY:
                cap = int(n.value)
                continue
            self._check(rc, "contacts")
            return ca.to_dict(int(n.value))

    def detect(self, tol: float, phase: int = 0) -> dict:
        return self._contacts(self._f("detect"), C.c_double(tol), C.c_int(phase))

    def constraints(self) -> dict:
        return self._contacts(self._f("get_constraints"))

    @property
    def dt(self) -> float:
        return self._f("get_dt")(self.h)

    @dt.setter
    def dt(self, v: float):
        self._f("set_dt")(self.h, v)

    @property
    def colony_radius(self) -> float:
        return self._f("colony_radius")(self.h)

    @property
    def division_count(self) -> int:
        return int(self._f("division_count")(self.h))


_REF_LIBS: dict = {}


class RefColony(_CpuColony):
    """The reference's own code (strict IEEE build unless fast=True)."""

    prefix = "pcc_ref_"

    def __init__(self, params: abi.Params, fast: bool = False, outdir: str | None = None):
        name = "libpccref_fast.so" if fast else "libpccref_strict.so"
        if name not in _REF_LIBS:
            lib = _load(name)
            _bind_common(lib, self.prefix)
            lib.pcc_ref_division_length.restype = C.c_double
            lib.pcc_ref_division_length.argtypes = [C.c_ulonglong, C.c_ulonglong, C.c_double]
            lib.pcc_ref_log_vtk.argtypes = [_VP, _P(abi.SimRecord)]
            lib.pcc_ref_load_vtk.argtypes = [C.c_char_p, _P(abi.Cells), C.c_size_t, _P(C.c_size_t),
                                             _P(C.c_double), _P(C.c_longlong), _P(C.c_double)]
            _REF_LIBS[name] = lib
        self.lib = _REF_LIBS[name]
        self.n_cells_hint = 1024
        self._tmp = tempfile.mkdtemp(prefix="pccref_") if outdir is None else outdir
        self._mode = params.mode
        self.h = self.lib.pcc_ref_create(C.byref(params), self._tmp.encode())


    @property
    def vtk_dir(self) -> Path:
        """Where the reference's loggers write (Domain's ./vtk_output_<mode>)."""
        return Path(self._tmp) / "vtk_output_hard" if self._mode == 0 else Path(self._tmp) / "vtk_output_soft"

    def log_vtk(self, record: abi.SimRecord):
        rc = self.lib.pcc_ref_log_vtk(self.h, C.byref(record))
        if rc != 0:
            raise RuntimeError("pcc_ref_log_vtk failed")


def ref_load_vtk(path: str):
    """The reference's VTKStateLoader on a directory: (cells, time, step, dt)."""
    if "libpccref_strict.so" not in _REF_LIBS:
        RefColony(abi.default_params())
    lib = _REF_LIBS["libpccref_strict.so"]
    n = C.c_size_t(0)
    t, dt = C.c_double(0), C.c_double(0)
    step = C.c_longlong(0)
    if lib.pcc_ref_load_vtk(str(path).encode(), None, 0, C.byref(n), C.byref(t), C.byref(step), C.byref(dt)):
        raise RuntimeError("reference loader failed")
    ca = abi.CellArrays(int(n.value))
    if lib.pcc_ref_load_vtk(str(path).encode(), C.byref(ca.struct), ca.cap, C.byref(n), C.byref(t), C.byref(step),
                            C.byref(dt)):
        raise RuntimeError("reference loader failed")
    return ca.to_dict(int(n.value)), t.value, int(step.value), dt.value


def ref_division_length(seed: int, k: int, length: float) -> float:
    if "libpccref_strict.so" not in _REF_LIBS:
        RefColony(abi.default_params())
    return _REF_LIBS["libpccref_strict.so"].pcc_ref_division_length(seed, k, length)


_ORACLE_LIB = None


class OracleColony(_CpuColony):
    """The plain-C restatement of the reference path."""

    prefix = "pcco_"

    def __init__(self, params: abi.Params):
        global _ORACLE_LIB
        if _ORACLE_LIB is None:
            lib = _load("libpcc_oracle.so")
            _bind_common(lib, self.prefix)
            lib.pcco_division_length.restype = C.c_double
            lib.pcco_division_length.argtypes = [C.c_ulonglong, C.c_ulonglong, C.c_double]
            lib.pcco_division_seed.restype = C.c_uint
            lib.pcco_division_seed.argtypes = [C.c_ulonglong, C.c_ulonglong]
            _ORACLE_LIB = lib
        self.lib = _ORACLE_LIB
        self.n_cells_hint = 1024
        self.h = self.lib.pcco_create(C.byref(params))


def oracle_division_length(seed: int, k: int, length: float) -> float:
    if _ORACLE_LIB is None:
        OracleColony(abi.default_params())
    return _ORACLE_LIB.pcco_division_length(seed, k, length)
