"""C-ABI checks that need no GPU: the device library loads, exports every
entry point include/pcc_gpu.h declares, and its host-side pieces (defaults,
division draws, argument checks) behave."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from helpers import load_fixture
from pcc_b200 import abi, device

HEADER = Path(__file__).resolve().parents[1] / "include" / "pcc_gpu.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pcc_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = device.load_library()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_default_params_match_reference_cli_defaults():
    lib = device.load_library()
    p = abi.Params()
    lib.pcc_default_params(C.byref(p))
    q = abi.default_params()
    for k, _ in abi.Params._fields_:
        assert getattr(p, k) == pytest.approx(getattr(q, k)), k
    assert p.linked_cell_size == 2.2 * p.l0
    assert p.tolerance == 1e-3 and p.max_bbpgd_iterations == 500000 and p.max_recursive_iterations == 50


def test_division_draws_of_device_code_match_libstdcxx():
    """The draw compiled for the device (host instantiation of the same
    function) equals std::mt19937 + std::uniform_real_distribution."""
    fx = load_fixture("division_draws")
    for seed, k, L, v in zip(fx["seed"], fx["k"], fx["length"], fx["value"]):
        assert device.division_length(int(seed), int(k), float(L)) == v


def test_create_rejects_bad_parameters():
    lib = device.load_library()
    h = C.c_void_p()
    p = abi.default_params(temperature=-1.0)
    assert lib.pcc_create(C.byref(p), 0, C.byref(h)) == abi.PCC_ERR_INVALID
    p = abi.default_params(mode=7)
    assert lib.pcc_create(C.byref(p), 0, C.byref(h)) == abi.PCC_ERR_INVALID
    p = abi.default_params(linked_cell_size=0.0)
    assert lib.pcc_create(C.byref(p), 0, C.byref(h)) == abi.PCC_ERR_INVALID
    p = abi.default_params(precision=7)
    assert lib.pcc_create(C.byref(p), 0, C.byref(h)) == abi.PCC_ERR_INVALID


def test_null_context_is_rejected():
    lib = device.load_library()
    st = abi.StepStats()
    assert lib.pcc_step(None, C.byref(st)) == abi.PCC_ERR_INVALID
    assert lib.pcc_solve(None, 1e-3, 0, C.byref(st)) == abi.PCC_ERR_INVALID
    assert lib.pcc_last_error(None) == b"null context"


def test_seed_cell_orientation_is_deterministic():
    a = abi.seed_cell(7)
    b = abi.seed_cell(7)
    assert a == b
    q = np.array([a["q0"][0], a["q1"][0], a["q2"][0], a["q3"][0]])
    assert abs(np.linalg.norm(q) - 1) < 1e-15 and q[1] == 0 and q[2] == 0
