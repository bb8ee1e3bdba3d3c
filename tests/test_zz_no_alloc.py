"""The allocation-free batched-chemistry entry point.

Some callers cannot let the library call cudaMalloc: an application that owns the device memory
budget through its own pool, or code that must not allocate between its setup and its launches.
ocfd_gpu_chem_batch_noalloc serves them by keeping its scratch in a fixed device array of the
library (at most 1048576 reactors). This test drives it through the C ABI on device buffers and
checks it against the allocating entry point, ocfd_gpu_chem_batch_device, on two calls in a row
(the second call reuses the array that the first one left behind), within the 1e-10 relative
tolerance of the chemistry parity tests.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _device(a):
    import torch
    return torch.tensor(a, device="cuda")


def test_noalloc_matches_allocating_entry_point():
    import torch

    from ocfd_b200 import abi, cases, solver
    names, th, kin, di, E, dt, nsub, T = cases.reactors(n=20000, seed=7)
    solver.chem_setup(th, kin, 1, abi.CHEM_IMPLICIT)
    L = solver.lib()
    n = len(E)
    cur_di, cur_e = di.copy(), E.copy()
    for call in range(2):
        a_di, a_e, a_dt, a_ns = _device(cur_di), _device(cur_e), _device(dt), _device(nsub)
        b_di, b_e, b_dt, b_ns = _device(cur_di), _device(cur_e), _device(dt), _device(nsub)
        solver.chem_batch_device(n, a_di.data_ptr(), a_e.data_ptr(), a_dt.data_ptr(), a_ns.data_ptr())
        rc = L.ocfd_gpu_chem_batch_noalloc(n, b_di.data_ptr(), b_e.data_ptr(), b_dt.data_ptr(), b_ns.data_ptr())
        assert rc == 0, L.ocfd_gpu_last_error().decode()
        torch.cuda.synchronize()
        ra, rb = a_di.cpu().numpy(), b_di.cpu().numpy()
        scale = np.abs(ra).max(axis=1, keepdims=True)
        assert (np.abs(ra - rb) / scale).max() <= TOL
        ea, eb = a_e.cpu().numpy(), b_e.cpu().numpy()
        assert np.abs(ea - eb).max() <= TOL * np.abs(ea).max()
        assert np.abs(ra - cur_di).max() > 0  # the reactors advanced
        cur_di, cur_e = ra.copy(), ea.copy()  # second call starts from the first call's result


def test_noalloc_rejects_oversized_batch():
    from ocfd_b200 import abi, cases, solver
    names, th, kin, *_ = cases.reactors(n=8, seed=0)
    solver.chem_setup(th, kin, 1, abi.CHEM_IMPLICIT)
    L = solver.lib()
    rc = L.ocfd_gpu_chem_batch_noalloc((1 << 20) + 1, None, None, None, None)
    assert rc == abi.ERR_PARAM
    assert "exceeds" in L.ocfd_gpu_last_error().decode()
