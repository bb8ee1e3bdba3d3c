"""The compiled H2-air mechanism kernels (ocfd_mech_h2air9.cuh, selected by
ocfd_gpu_chem_compiled_mechanism) against the generic kernels that read the mechanism from the
constant block: the same arithmetic with the zero terms left out, so both give the same bits on
the GPU (the batched reactors, constant volume and constant pressure, and the reacting jet's flow
step). The oracle comparisons of the other test files run the compiled kernels (the default for
this mechanism).
"""
import numpy as np
import pytest

from ocfd_b200 import abi, cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    from ocfd_b200 import solver
    solver.lib()
    return solver


def run_batch(gpu, compiled, const_p, n=1 << 16, seed=7):
    names, th, kin, di, E, dt, nsub, T = cases.reactors(n=n, seed=seed)
    gpu.chem_setup(th, kin, 1, abi.CHEM_IMPLICIT, const_p=const_p)
    used = gpu.lib().ocfd_gpu_chem_compiled_mechanism(1 if compiled else 0)
    d, e = di.copy(), E.copy()
    gpu.chem_batch(d, e, dt, nsub)
    gpu.lib().ocfd_gpu_chem_compiled_mechanism(1)
    if const_p:
        gpu.lib().ocfd_gpu_chem_constant_pressure(0)
    return used, d, e, di


@pytest.mark.parametrize("const_p", [False, True], ids=["constant_volume", "constant_pressure"])
def test_compiled_mechanism_equals_generic_batch(gpu, const_p):
    used_c, dc, ec, di = run_batch(gpu, True, const_p)
    used_g, dg, eg, _ = run_batch(gpu, False, const_p)
    assert used_c == 1 and used_g == 0
    assert np.array_equal(dc, dg)
    assert np.array_equal(ec, eg)
    assert np.abs(dc - di).max() > 0  # the reactors advanced


def test_compiled_mechanism_equals_generic_flow_step(gpu):
    c = cases.jet(nx=24, ny=16, nz=16)
    out = []
    for compiled in (1, 0):
        g = gpu.Solver(c)
        assert gpu.lib().ocfd_gpu_chem_compiled_mechanism(compiled) == compiled
        g.init_state()
        for s in range(3):
            g.tt = s * c.dt
            g.step(c.dt, 1, 1)
        out.append(g.download_state())
        g.close()
    (fa, da, pa), (fb, db, pb) = out
    assert np.array_equal(fa, fb)
    assert np.array_equal(da, db)
    assert np.array_equal(pa, pb)


def test_other_structure_keeps_generic_kernels(gpu):
    names, th, kin, *_ = cases.reactors(n=64, seed=1)
    gpu.chem_setup(th, kin, 1, abi.CHEM_IMPLICIT)
    assert gpu.lib().ocfd_gpu_chem_compiled_mechanism(-1) == 1
    kin.vr[3][4] = 1  # O + H2O = OH (a different stoichiometry): not the compiled mechanism
    gpu.chem_setup(th, kin, 1, abi.CHEM_IMPLICIT)
    assert gpu.lib().ocfd_gpu_chem_compiled_mechanism(-1) == 0
    names, th, kin, *_ = cases.reactors(n=64, seed=1)
    gpu.chem_setup(th, kin, 1, abi.CHEM_RK3)  # the compiled kernels carry the implicit step only
    assert gpu.lib().ocfd_gpu_chem_compiled_mechanism(-1) == 0
    gpu.chem_setup(th, kin, 1, abi.CHEM_IMPLICIT)
    assert gpu.lib().ocfd_gpu_chem_compiled_mechanism(-1) == 1
