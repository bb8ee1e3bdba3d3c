"""The allocation-free batched-chemistry entry point.

Some callers cannot let the library call cudaMalloc: an application that owns the device memory
budget through its own pool, or code that must not allocate between its setup and its launches.
ocfd_gpu_chem_batch_noalloc serves them by keeping its scratch in a fixed device array of the
library (at most 1048576 reactors). This test drives it through the C ABI on device buffers and
checks it against the allocating entry point, ocfd_gpu_chem_batch_device, on two calls in a row
(the second call reuses the array that the first one left behind). Both entry points run the same
kernel on every reactor, so the results must be equal bit for bit. The no-alloc call runs first in
each round, and the device's free memory must not change across the second one.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


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
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        rc = L.ocfd_gpu_chem_batch_noalloc(n, b_di.data_ptr(), b_e.data_ptr(), b_dt.data_ptr(), b_ns.data_ptr())
        assert rc == 0, L.ocfd_gpu_last_error().decode()
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info()[0]
        if call == 1:  # the first call may load the library's kernels; the second allocates nothing
            assert free1 == free0, (free0, free1)
        solver.chem_batch_device(n, a_di.data_ptr(), a_e.data_ptr(), a_dt.data_ptr(), a_ns.data_ptr())
        torch.cuda.synchronize()
        ra, rb = a_di.cpu().numpy(), b_di.cpu().numpy()
        ea, eb = a_e.cpu().numpy(), b_e.cpu().numpy()
        assert np.array_equal(ra, rb)
        assert np.array_equal(ea, eb)
        assert np.abs(ra - cur_di).max() > 0  # the reactors advanced
        cur_di, cur_e = ra.copy(), ea.copy()  # second call starts from the first call's result


def test_noalloc_rejects_oversized_and_negative_batches():
    from ocfd_b200 import abi, cases, solver
    names, th, kin, *_ = cases.reactors(n=8, seed=0)
    solver.chem_setup(th, kin, 1, abi.CHEM_IMPLICIT)
    L = solver.lib()
    rc = L.ocfd_gpu_chem_batch_noalloc((1 << 20) + 1, None, None, None, None)
    assert rc == abi.ERR_PARAM
    assert "exceeds" in L.ocfd_gpu_last_error().decode()
    rc = L.ocfd_gpu_chem_batch_noalloc(-1, None, None, None, None)
    assert rc == abi.ERR_PARAM
    assert "must be >= 0" in L.ocfd_gpu_last_error().decode()
    assert L.ocfd_gpu_chem_batch_noalloc(0, None, None, None, None) == 0
