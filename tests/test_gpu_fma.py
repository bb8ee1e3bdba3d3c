"""The contracted multiply-add build (libocfd_gpu_fma.so, `make -C opencfd-comb_b200 fma`)
against the CPU oracle under the hot path's tolerance: ten full steps on each configuration's
physics, relative L-infinity <= 1e-10 on every conserved variable and species density, and the
HYBRID decision maps identical after every step. The variant runs in a child process
(tests/fma_child.py), the oracle here.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from ocfd_b200 import abi, solver

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
L = 4
TOL = 1e-10
FMA_LIB = os.path.join(os.path.dirname(solver.LIBPATH), "libocfd_gpu_fma.so")


def interior(a):
    return a[..., L:-L, L:-L, L:-L]


def rel_linf(a, b):
    den = np.abs(a).max()
    return float(np.abs(a - b).max() / (den if den > 0 else 1.0))


def decisions(c, rh):
    th1, th2 = c.params.hybrid_para[1], c.params.hybrid_para[2]
    r = interior(rh)
    out = []
    for ax in (2, 1, 0):
        a = np.moveaxis(r, ax, -1)
        out.append(np.digitize(np.maximum(a[..., :-1], a[..., 1:]), [th1, th2], right=True))
    return out


@pytest.fixture(scope="module")
def fma_results(tmp_path_factory):
    if not os.path.exists(FMA_LIB):
        pytest.fail("libocfd_gpu_fma.so is not built (make -C opencfd-comb_b200 fma)")
    d = tmp_path_factory.mktemp("fma")
    sys.path.insert(0, HERE)
    import fma_child
    env = dict(os.environ, OCFD_B200_LIB="fma")
    subprocess.check_call([sys.executable, os.path.join(HERE, "fma_child.py"), str(d)] +
                          list(fma_child.protocol_cases()), env=env, timeout=600)
    return d, fma_child.protocol_cases()


@pytest.mark.parametrize("name", ["isotropic16_weno5", "flatplate_hybrid", "flatplate_omp6", "jet24"])
def test_fma_build_within_tolerance(oracle, fma_results, name):
    d, table = fma_results
    z = np.load(os.path.join(str(d), name + ".npz"))
    assert str(z["variant"]) == "fma"
    builder, steps, ifr, nsub = table[name]
    c = builder()
    o = oracle.OracleSolver(c)
    o.init_state()
    for s in range(steps):
        o.step(c.dt, s * c.dt, ifr, nsub)
        if c.params.scheme_invis == abi.SCHEME_HYBRID:
            for mo, mg in zip(decisions(c, o.rhybrid()), decisions(c, z["rh"][s])):
                assert np.array_equal(mo, mg), "HYBRID decisions differ at step %d" % (s + 1)
    fo, dio, pro = o.download_state()
    o.close()
    for m in range(5):
        assert rel_linf(fo[m], z["f"][m]) <= TOL, (m, rel_linf(fo[m], z["f"][m]))
    for m in range(dio.shape[0]):
        assert rel_linf(interior(dio[m]), interior(z["di"][m])) <= TOL
    assert rel_linf(interior(pro[4]), interior(z["prims"][4])) <= TOL
