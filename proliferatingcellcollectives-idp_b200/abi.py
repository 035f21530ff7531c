"""ctypes mirror of include/pcc_gpu.h (the C ABI of the device library).

The structures here are byte-for-byte the ones declared in the header; the
host-side helpers turn numpy SoA arrays into the pointer structs the ABI takes.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

PCC_OK = 0
PCC_ERR_INVALID = 1
PCC_ERR_NOCONV_BBPGD = 2
PCC_ERR_NOCONV_RELCP = 3
PCC_ERR_CAPACITY = 4
PCC_ERR_TIMEOUT = 5
PCC_ERR_BOUNDS = 6
PCC_ERR_CUDA = 7
PCC_ERR_NAN = 8
PCC_ERR_NOMEM = 9

STATUS_NAMES = {
    0: "PCC_OK", 1: "PCC_ERR_INVALID", 2: "PCC_ERR_NOCONV_BBPGD", 3: "PCC_ERR_NOCONV_RELCP",
    4: "PCC_ERR_CAPACITY", 5: "PCC_ERR_TIMEOUT", 6: "PCC_ERR_BOUNDS", 7: "PCC_ERR_CUDA",
    8: "PCC_ERR_NAN", 9: "PCC_ERR_NOMEM",
}

MODE_HARD = 0
MODE_SOFT = 1
GHOSTS_NONE = 0
GHOSTS_SINGLE_RANK = 1
PRECISION_FP64 = 0
PRECISION_MIXED = 1
SOLVER_AUTO = 0
SOLVER_GENERAL = 1

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class Params(C.Structure):
    _fields_ = [
        ("dt", C.c_double),
        ("end_radius", C.c_double),
        ("xi", C.c_double),
        ("tau", C.c_double),
        ("l0", C.c_double),
        ("lambda_", C.c_double),
        ("temperature", C.c_double),
        ("kcc", C.c_double),
        ("monolayer", C.c_int),
        ("tolerance", C.c_double),
        ("max_bbpgd_iterations", C.c_longlong),
        ("max_recursive_iterations", C.c_longlong),
        ("linked_cell_size", C.c_double),
        ("cfl_factor", C.c_double),
        ("mode", C.c_int),
        ("fixed_dt", C.c_int),
        ("dt_cap", C.c_double),
        ("ghost_mode", C.c_int),
        ("seed", C.c_ulonglong),
        ("precision", C.c_int),
        ("capacity_hint", C.c_longlong),
        ("solver_variant", C.c_int),
        ("log_every_colony_radius_delta", C.c_double),
        ("log_every_sim_time_delta", C.c_double),
        ("log_bbpgd_trace", C.c_int),
    ]


class Cells(C.Structure):
    _fields_ = [(n, _dp) for n in ("x", "y", "z", "q0", "q1", "q2", "q3", "length", "l0", "diameter",
                                   "ldot", "impedance", "stress")] + [("age", _ip), ("force", _dp),
                                                                      ("velocity", _dp),
                                                                      ("num_constraints", _ip)]


class Contacts(C.Structure):
    _fields_ = [("gid_i", _ip), ("gid_j", _ip), ("sd", _dp), ("normal", _dp), ("r_i", _dp), ("r_j", _dp),
                ("contact_point", _dp), ("stress_i", _dp), ("stress_j", _dp), ("gamma", _dp), ("phase", _ip)]


class StepStats(C.Structure):
    _fields_ = [
        ("relcp_iterations", C.c_int),
        ("bbpgd_iterations", C.c_longlong),
        ("residual", C.c_double),
        ("max_overlap", C.c_double),
        ("n_constraints", C.c_longlong),
        ("n_cells", C.c_longlong),
        ("n_divided", C.c_longlong),
        ("dt_used", C.c_double),
        ("dt_next", C.c_double),
        ("colony_radius", C.c_double),
        ("sim_time", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Profile(C.Structure):
    _fields_ = [
        ("bbpgd_launches", C.c_longlong),
        ("bbpgd_iterations", C.c_longlong),
        ("bbpgd_ms", C.c_double),
        ("bbpgd_algo_bytes", C.c_double),
        ("detect_ms", C.c_double),
        ("solve_ms", C.c_double),
        ("solves", C.c_longlong),
        ("cell_solves", C.c_double),
        ("detect_full_passes", C.c_longlong),
        ("detect_list_passes", C.c_longlong),
        ("bbpgd_grid_launches", C.c_longlong),
        ("bbpgd_cta_launches", C.c_longlong),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Job(C.Structure):
    _fields_ = [("params", Params), ("end_radius", C.c_double), ("arrival_s", C.c_double),
                ("max_steps", C.c_longlong)]


class JobResult(C.Structure):
    _fields_ = [
        ("status", C.c_int),
        ("steps", C.c_longlong),
        ("cells", C.c_longlong),
        ("cell_steps", C.c_double),
        ("bbpgd_iterations", C.c_longlong),
        ("arrival_s", C.c_double),
        ("start_s", C.c_double),
        ("finish_s", C.c_double),
        ("footprint_bytes", C.c_double),
        ("checksum", C.c_double),
        ("max_step_bbpgd", C.c_longlong),
        ("radius", C.c_double),
        ("dt", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class TraceStep(C.Structure):
    _fields_ = [("step", C.c_ulonglong), ("recursive_iteration", C.c_ulonglong), ("total_constraints", C.c_ulonglong),
                ("residual", C.c_double), ("step_size", C.c_double), ("linear", C.c_double),
                ("quadratic", C.c_double), ("growth", C.c_double), ("total", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class SimRecord(C.Structure):
    _fields_ = [
        ("simulation_time_s", C.c_double),
        ("time_since_last_log_s", C.c_double),
        ("step", C.c_ulonglong),
        ("num_particles", C.c_int),
        ("num_constraints", C.c_ulonglong),
        ("colony_radius", C.c_double),
        ("recursive_iterations", C.c_int),
        ("bbpgd_iterations", C.c_ulonglong),
        ("max_overlap", C.c_double),
        ("residual", C.c_double),
        ("dt_s", C.c_double),
        ("memory_usage_mb", C.c_double),
        ("peak_memory_mb", C.c_double),
        ("cpu_time_s", C.c_double),
        ("mpi_comm_time_s", C.c_double),
        ("load_imbalance", C.c_double),
    ]


def default_params(**over) -> Params:
    """Reference defaults (code/cpp/src/util/CLIParser.h:296-365), hard mode."""
    p = Params()
    p.dt = 1e-2
    p.end_radius = 50.0
    p.xi = 1.0
    p.tau = 1.0
    p.l0 = 1.0
    p.lambda_ = 1e-2
    p.temperature = 0.0
    p.kcc = 20000.0
    p.monolayer = 1
    p.tolerance = 1e-3
    p.max_bbpgd_iterations = 500000
    p.max_recursive_iterations = 50
    p.linked_cell_size = 2.2 * p.l0
    p.cfl_factor = 0.5
    p.mode = MODE_HARD
    p.fixed_dt = 0
    p.dt_cap = 0.0
    p.ghost_mode = GHOSTS_SINGLE_RANK
    p.seed = 0
    p.precision = 0
    p.capacity_hint = 0
    p.solver_variant = 0
    p.log_every_colony_radius_delta = 0.5
    p.log_every_sim_time_delta = 100000.0
    for k, v in over.items():
        if k == "lambda":
            k = "lambda_"
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


CELL_FIELDS = ("x", "y", "z", "q0", "q1", "q2", "q3", "length", "l0", "diameter", "ldot", "impedance",
               "stress")


class CellArrays:
    """Host SoA buffers of `cap` cells plus the Cells pointer struct over them."""

    def __init__(self, cap: int):
        self.cap = int(cap)
        self.arrays = {f: np.zeros(max(self.cap, 1), np.float64) for f in CELL_FIELDS}
        self.arrays["age"] = np.zeros(max(self.cap, 1), np.int32)
        self.arrays["force"] = np.zeros(6 * max(self.cap, 1), np.float64)
        self.arrays["velocity"] = np.zeros(6 * max(self.cap, 1), np.float64)
        self.arrays["num_constraints"] = np.zeros(max(self.cap, 1), np.int32)
        self.struct = Cells()
        for f in CELL_FIELDS + ("force", "velocity"):
            setattr(self.struct, f, self.arrays[f].ctypes.data_as(_dp))
        self.struct.age = self.arrays["age"].ctypes.data_as(_ip)
        self.struct.num_constraints = self.arrays["num_constraints"].ctypes.data_as(_ip)

    @classmethod
    def from_dict(cls, cells: dict) -> "CellArrays":
        n = len(cells["x"])
        ca = cls(n)
        for k, v in cells.items():
            if k in ca.arrays:
                a = np.asarray(v)
                ca.arrays[k][: a.size] = a.reshape(-1)
        return ca

    def to_dict(self, n: int) -> dict:
        out = {f: self.arrays[f][:n].copy() for f in CELL_FIELDS + ("age", "num_constraints")}
        out["force"] = self.arrays["force"][: 6 * n].reshape(n, 6).copy()
        out["velocity"] = self.arrays["velocity"][: 6 * n].reshape(n, 6).copy()
        return out


CONTACT_FIELDS_INT = ("gid_i", "gid_j", "phase")
CONTACT_FIELDS_1 = ("sd", "stress_i", "stress_j", "gamma")
CONTACT_FIELDS_3 = ("normal", "r_i", "r_j", "contact_point")


class ContactArrays:
    def __init__(self, cap: int):
        self.cap = int(cap)
        c = max(self.cap, 1)
        self.arrays = {f: np.zeros(c, np.int32) for f in CONTACT_FIELDS_INT}
        self.arrays.update({f: np.zeros(c, np.float64) for f in CONTACT_FIELDS_1})
        self.arrays.update({f: np.zeros(3 * c, np.float64) for f in CONTACT_FIELDS_3})
        self.struct = Contacts()
        for f in CONTACT_FIELDS_INT:
            setattr(self.struct, f, self.arrays[f].ctypes.data_as(_ip))
        for f in CONTACT_FIELDS_1 + CONTACT_FIELDS_3:
            setattr(self.struct, f, self.arrays[f].ctypes.data_as(_dp))

    def to_dict(self, n: int) -> dict:
        out = {f: self.arrays[f][:n].copy() for f in CONTACT_FIELDS_INT + CONTACT_FIELDS_1}
        out.update({f: self.arrays[f][: 3 * n].reshape(n, 3).copy() for f in CONTACT_FIELDS_3})
        return out


def seed_cell(seed: int, l0: float = 1.0) -> dict:
    """The first cell of a colony: centre at the origin, diameter l0/2, length
    l0 (code/cpp/src/main.cpp:27-30), orientation theta ~ U[0, pi) drawn from
    `seed` (q = (cos theta/2, 0, 0, sin theta/2), rotation about z)."""
    theta = float(np.random.default_rng(seed).uniform(0.0, np.pi))
    return {
        "x": [0.0], "y": [0.0], "z": [0.0],
        "q0": [np.cos(theta / 2)], "q1": [0.0], "q2": [0.0], "q3": [np.sin(theta / 2)],
        "length": [l0], "l0": [l0], "diameter": [l0 / 2], "age": [1],
    }
