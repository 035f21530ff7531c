"""pcc_soft_forces_noalloc: the soft-model force assembly for callers that
must not let the library allocate device memory (a host that accounts its HBM
through its own fixed pool, or a loop sharing the GPU with other colonies'
streams where cudaFree's device-wide wait would stall them).

The caller owns every device buffer (allocated here through torch); the
entry point's intermediates live in its fixed device scratch array.  Its
output must match the force assembly of the existing entry point
(pcc_soft_forces_frozen) within the soft-model tolerance of the parity tests,
on two calls in a row -- the second call reuses the scratch the first one
left behind.  This file is collected last (test_zz_*) so a failure here
cannot hide another test's result; it passes alone and after the others.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from helpers import load_fixture, params_of, sub
from pcc_b200 import abi
from pcc_b200.device import Colony, load_library

pytestmark = pytest.mark.gpu

MAX_CELLS = 65536
MAX_CONTACTS = 393216


def _entry():
    f = load_library().pcc_soft_forces_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p] * 8 + [C.c_size_t, C.c_void_p, C.c_size_t, C.c_double, C.c_void_p, C.c_void_p,
                                     C.c_void_p]
    return f


@pytest.mark.parametrize("name", ["soft_on_hard_r10_seed3", "hard_r10_seed3"])
def test_noalloc_soft_forces_match_existing_entry_point(name):
    import torch

    f = _entry()
    fx = load_fixture(name)
    p = params_of(fx, mode=abi.MODE_SOFT, kcc=1333.3333333333333)
    cells = sub(fx, "cells_")
    col = Colony(p)
    col.set_cells(cells)
    contacts = col.detect(0.0)
    col.soft_forces_frozen(1)  # existing entry point: force and stress into the resident cells
    want = col.get_cells()
    n, m = len(cells["x"]), contacts["sd"].size
    assert 0 < m <= MAX_CONTACTS and n <= MAX_CELLS

    dev = torch.device("cuda:0")

    def t(a, dtype):
        return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=dev)

    gi, gj = t(contacts["gid_i"], torch.int32), t(contacts["gid_j"], torch.int32)
    sd = t(contacts["sd"], torch.float64)
    normal, ri, rj = (t(contacts[k].reshape(-1), torch.float64) for k in ("normal", "r_i", "r_j"))
    si, sj = t(contacts["stress_i"], torch.float64), t(contacts["stress_j"], torch.float64)
    diam = t(cells["diameter"], torch.float64)
    force = torch.empty(6 * n, dtype=torch.float64, device=dev)
    stress = torch.empty(n, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):  # two calls in a row on the shared scratch
        force.fill_(float("nan"))
        stress.fill_(float("nan"))
        torch.cuda.synchronize(dev)
        # the first call on a device may load the module (driver memory); a
        # warm call must not change the device's free memory or torch's pool
        free0, torch0 = torch.cuda.mem_get_info(dev)[0], torch.cuda.memory_allocated(dev)
        rc = f(gi.data_ptr(), gj.data_ptr(), sd.data_ptr(), normal.data_ptr(), ri.data_ptr(), rj.data_ptr(),
               si.data_ptr(), sj.data_ptr(), m, diam.data_ptr(), n, p.kcc, force.data_ptr(), stress.data_ptr(),
               stream)
        torch.cuda.synchronize(dev)
        assert rc == abi.PCC_OK
        if call == 1:
            assert torch.cuda.mem_get_info(dev)[0] == free0
            assert torch.cuda.memory_allocated(dev) == torch0
        np.testing.assert_allclose(force.cpu().numpy().reshape(n, 6), want["force"], rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(stress.cpu().numpy(), want["stress"], rtol=1e-12, atol=1e-12)


def test_noalloc_skips_and_reports_out_of_range_ids():
    """A contact naming a cell id >= n is skipped on the device (nothing is
    written for it) and the call returns PCC_ERR_BOUNDS; the other contacts
    give exactly the assembly of the list without it."""
    import torch

    f = _entry()
    fx = load_fixture("soft_on_hard_r10_seed3")
    p = params_of(fx)
    cells = sub(fx, "cells_")
    col = Colony(p)
    col.set_cells(cells)
    c = col.detect(0.0)
    n, m = len(cells["x"]), c["sd"].size
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev).cuda_stream
    bad = int(np.argmin(c["sd"]))  # an overlapping contact, so it would carry a force

    def run(keep, gj):
        def t(a, dtype):
            return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=dev)
        args = [t(c["gid_i"][keep], torch.int32), t(gj[keep], torch.int32), t(c["sd"][keep], torch.float64)]
        args += [t(c[k][keep].reshape(-1), torch.float64) for k in ("normal", "r_i", "r_j")]
        args += [t(c["stress_i"][keep], torch.float64), t(c["stress_j"][keep], torch.float64)]
        diam = t(cells["diameter"], torch.float64)
        force = torch.full((6 * n,), float("nan"), dtype=torch.float64, device=dev)
        stress = torch.full((n,), float("nan"), dtype=torch.float64, device=dev)
        rc = f(*[a.data_ptr() for a in args], int(keep.sum()), diam.data_ptr(), n, p.kcc, force.data_ptr(),
               stress.data_ptr(), stream)
        torch.cuda.synchronize(dev)
        return rc, force.cpu().numpy(), stress.cpu().numpy()

    every = np.ones(m, dtype=bool)
    without = every.copy()
    without[bad] = False
    gj_bad = c["gid_j"].copy()
    gj_bad[bad] = n + 5
    rc0, f0, s0 = run(without, c["gid_j"])
    rc1, f1, s1 = run(every, gj_bad)
    assert rc0 == abi.PCC_OK and rc1 == abi.PCC_ERR_BOUNDS
    np.testing.assert_array_equal(f1, f0)
    np.testing.assert_array_equal(s1, s0)
    gj_bad[bad] = -1
    rc2, f2, _ = run(every, gj_bad)
    assert rc2 == abi.PCC_ERR_BOUNDS
    np.testing.assert_array_equal(f2, f0)
    rc3, f3, _ = run(every, c["gid_j"])  # the flag does not outlive the call
    assert rc3 == abi.PCC_OK


def test_noalloc_rejects_sizes_beyond_its_scratch():
    f = _entry()
    assert f(None, None, None, None, None, None, None, None, MAX_CONTACTS + 1, None, 10, 1.0, None, None,
             None) == abi.PCC_ERR_CAPACITY
    assert f(None, None, None, None, None, None, None, None, 0, None, MAX_CELLS + 1, 1.0, None, None,
             None) == abi.PCC_ERR_CAPACITY
