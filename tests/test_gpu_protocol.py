"""The correctness protocol of the hot path, on the GPU through the C ABI against the CPU oracle:
ten full time steps on identical seeded inputs for each configuration's physics, with the
hybrid-scheme decision maps compared step by step; the hybrid sensor's second form (|grad p|
over its global mean) with forced patches; the mass-force source; the error paths the reference
stops on; the committed golden fixtures; the batched reactors at their full configured size.

Bitwise where no transcendental function enters (perfect / NASA-fit gas, Sutherland transport,
every reconstruction), <= 1e-10 relative L-infinity after ten steps where exp / log / pow do
(Wilke transport, finite-rate chemistry).
"""
import os

import numpy as np
import pytest

from ocfd_b200 import abi, cases

pytestmark = pytest.mark.gpu
L = 4
TOL = 1e-10
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def gpu():
    from ocfd_b200 import solver
    solver.lib()
    return solver


def interior(a):
    return a[..., L:-L, L:-L, L:-L]


def rel_linf(a, b):
    den = np.abs(a).max()
    return float(np.abs(a - b).max() / (den if den > 0 else 1.0))


def decisions(c, rh):
    """Per-interface scheme of HYBRID in each direction: R = max(R_i, R_i+1) against theta1 / theta2
    (OCFD_Schemes.f90:329-370, set_hybrid_scheme OCFD_SetHybrid.f90:2-15); 0 = UD7L, 1 = WENO7,
    2 = WENO5."""
    th1, th2 = c.params.hybrid_para[1], c.params.hybrid_para[2]
    r = interior(rh)
    out = []
    for ax in (2, 1, 0):  # i, j, k of the (k, j, i) array
        a = np.moveaxis(r, ax, -1)
        R = np.maximum(a[..., :-1], a[..., 1:])
        out.append(np.digitize(R, [th1, th2], right=True))
    return out


def run10(oracle, gpu, case, nsteps=10, if_reaction=0, nsub=1, track_hybrid=False):
    """nsteps Strang steps on the oracle and on the GPU; the hybrid decision maps of every step
    (they are set at the first stage of each flow half-step) are compared as the run goes."""
    o = oracle.OracleSolver(case)
    o.init_state()
    g = gpu.Solver(case)
    g.init_state()
    maps_checked = 0
    for s in range(nsteps):
        tt = s * case.dt
        o.step(case.dt, tt, if_reaction, nsub)
        g.tt = tt
        g.step(case.dt, if_reaction, nsub)
        if track_hybrid:
            ro, rg = o.rhybrid(), g.rhybrid()
            for mo, mg in zip(decisions(case, ro), decisions(case, rg)):
                assert np.array_equal(mo, mg), "hybrid decisions differ at step %d" % (s + 1)
            maps_checked += 1
    so, sg = o.download_state(), g.download_state()
    o.close()
    g.close()
    return so, sg, maps_checked


def assert_bitwise(so, sg):
    fo, dio, pro = so
    fg, dig, prg = sg
    assert np.array_equal(fo, fg), [rel_linf(fo[m], fg[m]) for m in range(5)]
    assert np.array_equal(interior(pro), interior(prg))
    assert np.array_equal(interior(dio), interior(dig))


def assert_close(so, sg, ns):
    fo, dio, pro = so
    fg, dig, prg = sg
    for m in range(5):
        assert rel_linf(fo[m], fg[m]) <= TOL, (m, rel_linf(fo[m], fg[m]))
    for m in range(ns):
        e = rel_linf(interior(dio[m]), interior(dig[m]))
        assert e <= TOL, (m, e)
    assert rel_linf(interior(pro[4]), interior(prg[4])) <= TOL


# ---------------------------------------------------------------- ten steps per configuration
def test_ten_steps_isotropic_weno5_cd6(oracle, gpu):
    """C1 physics: periodic box, WENO5 Steger-Warming, CD6 viscous terms, Sutherland."""
    c = cases.isotropic(n=16)
    so, sg, _ = run10(oracle, gpu, c)
    assert_bitwise(so, sg)


def test_ten_steps_flatplate_hybrid_maps(oracle, gpu):
    """C2 physics: HYBRID UD7L / WENO7 / WENO5 with shock sensor 1, boundary-layer boundary
    conditions with the wall disturbance; decision maps identical after every step."""
    c = cases.flatplate(nx=40, ny=24, nz=12, scheme="HYBRID", lx=0.01, ly=0.004, y1=2e-5)
    so, sg, n = run10(oracle, gpu, c, track_hybrid=True)
    assert n == 10
    assert_bitwise(so, sg)


def test_ten_steps_flatplate_omp6(oracle, gpu):
    """C2 physics with OMP6 (its MP-limiter switch decisions are part of the bitwise state)."""
    c = cases.flatplate(nx=40, ny=24, nz=12, scheme="OMP6", lx=0.01, ly=0.004, y1=2e-5)
    so, sg, _ = run10(oracle, gpu, c)
    assert_bitwise(so, sg)


def test_ten_steps_reacting_jet(oracle, gpu):
    """C5 physics: 9-species H2 jet, WENO5, CD6, Wilke transport, implicit chemistry."""
    c = cases.jet(nx=24, ny=16, nz=16)
    so, sg, _ = run10(oracle, gpu, c, if_reaction=1, nsub=c.nsub)
    assert_close(so, sg, 9)


def test_ten_steps_reacting_box_two_substeps(oracle, gpu):
    """Hot 9-species mixture (T = 1500 K) where the chemistry changes the state every step."""
    names, *_ = cases.h2air_structs()
    Y = [1e-6, 0.2, 0.02, 0.1, 1e-5, 1e-6, 1e-7, 1e-7, 0.68]
    c = cases.isotropic(n=12, species=names, Y=Y, wilke=True, T0=1500.0)
    so, sg, _ = run10(oracle, gpu, c, if_reaction=1, nsub=2)
    assert_close(so, sg, 9)


# ---------------------------------------------------------------- hybrid sensor 2 and patches
def test_hybrid_sensor2_with_forced_patches(oracle, gpu):
    """comput_Rhybrid's second sensor, |grad p| over its global mean (OCFD_SetHybrid.f90:44-78),
    and two forced patches (:80-102). The mean is a sum over every cell, taken in a different
    order on the GPU, so Rhybrid agrees to rounding; every decision and the state are identical."""
    c = cases.flatplate(nx=40, ny=24, nz=12, scheme="HYBRID", lx=0.01, ly=0.004, y1=2e-5)
    hp = c.params.hybrid_para
    hp[0] = 2.0
    hp[1], hp[2] = 0.8, 2.5  # thresholds on the normalised gradient: all three schemes occur
    hp[3] = 2.0
    hp[4:10] = [3, 9, 1, 6, 2, 5]
    hp[10:16] = [20, 30, 10, 20, 1, 12]
    o = oracle.OracleSolver(c)
    o.init_state()
    g = gpu.Solver(c)
    g.init_state()
    used = set()
    for s in range(4):
        o.step(c.dt, s * c.dt)
        g.tt = s * c.dt
        g.step(c.dt)
        ro, rg = o.rhybrid(), g.rhybrid()
        assert rel_linf(interior(ro), interior(rg)) <= 1e-13
        for mo, mg in zip(decisions(c, ro), decisions(c, rg)):
            assert np.array_equal(mo, mg)
            used |= set(np.unique(mg).tolist())
        # the patches hold Rhybrid >= 100 (the most robust scheme) inside their boxes
        r = interior(rg)
        assert r[1:5, 0:6, 2:9].min() >= 100.0 and r[0:12, 9:20, 19:30].min() >= 100.0
    assert used == {0, 1, 2}  # UD7L, WENO7 and WENO5 interfaces all occur
    assert_bitwise(o.download_state(), g.download_state())
    o.close()
    g.close()


# ---------------------------------------------------------------- mass force
def test_mass_force_bitwise(oracle, gpu):
    """IF_Mass_Force = 1: du(2..4) += d f, du(5) += d (u . f) (OCFD_inviscous.f90:187-199)."""
    c = cases.isotropic(n=12)
    c.params.if_mass_force = 1
    c.params.mass_force[0], c.params.mass_force[1], c.params.mass_force[2] = 3.0e4, -1.5e4, 7.0e3
    so, sg, _ = run10(oracle, gpu, c, nsteps=3)
    assert_bitwise(so, sg)
    # and the force acts: the mean x-momentum differs from the run without it
    c0 = cases.isotropic(n=12)
    g = gpu.Solver(c0)
    g.init_state()
    for s in range(3):
        g.tt = s * c0.dt
        g.step(c0.dt)
    f0, _, _ = g.download_state()
    g.close()
    assert abs(sg[0][1].mean() - f0[1].mean()) > 1e-6 * np.abs(f0[1]).max()


# ---------------------------------------------------------------- error paths
def test_nan_state_is_reported(gpu):
    """A NaN in the uploaded conserved state stops the step with OCFD_ERR_NAN (the reference's
    debug_NaN stop, OCFD_debug.f90:20-26), it does not propagate silently."""
    c = cases.isotropic(n=12)
    g = gpu.Solver(c)
    g.init_state()
    f, di, pr = g.download_state()
    f[4, 3, 4, 5] = np.nan
    pr[6, L + 3, L + 4, L + 5] = np.nan
    g.upload_state(f, di, pr)
    with pytest.raises(gpu.OcfdError) as ei:
        g.step(c.dt)
    assert ei.value.code == abi.ERR_NAN
    g.close()


def test_bad_reactors_are_reported(gpu):
    """Batched chemistry: a reactor with no mass (every density zero) or a non-finite energy gives
    OCFD_ERR_CHEM instead of silent NaNs; the other reactors are still integrated as usual."""
    names, th, kin, di, E, dt, nsub, T = cases.reactors(n=256, seed=5)
    gpu.chem_setup(th, kin, 1, abi.CHEM_IMPLICIT)
    good_di, good_e = di.copy(), E.copy()
    gpu.chem_batch(good_di, good_e, dt, nsub)
    bad_di, bad_e = di.copy(), E.copy()
    bad_di[17] = 0.0
    bad_e[17] = 0.0
    bad_e[200] = np.nan
    with pytest.raises(gpu.OcfdError) as ei:
        gpu.chem_batch(bad_di, bad_e, dt, nsub)
    assert ei.value.code == abi.ERR_CHEM
    import ctypes as C
    nf, nb = C.c_longlong(), C.c_longlong()
    assert gpu.lib().ocfd_gpu_chem_batch_status(C.byref(nf), C.byref(nb)) == 0
    assert nb.value == 2
    keep = np.ones(256, bool)
    keep[[17, 200]] = False
    assert np.array_equal(bad_di[keep], good_di[keep]) and np.array_equal(bad_e[keep], good_e[keep])


# ---------------------------------------------------------------- golden fixtures
GOLDEN_EXACT = {"isotropic12_weno5", "isotropic12_omp6", "flatplate_hybrid", "isotropic10_o2n2"}


@pytest.mark.parametrize("name", ["isotropic12_weno5", "isotropic12_omp6", "flatplate_hybrid", "isotropic10_o2n2",
                                  "isotropic8_h2air"])
def test_gpu_matches_golden_fixture(gpu, name):
    """The CUDA path against the committed fixtures of tests/golden/ (written by make_golden.py
    with the oracle): bit for bit where no transcendental function enters, 1e-10 otherwise."""
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_golden
    builder, steps, ifr, nsub = make_golden.golden_cases()[name]
    z = np.load(os.path.join(HERE, "golden", name + ".npz"))
    c = builder()
    assert c.dt == float(z["dt"])
    g = gpu.Solver(c)
    g.init_state()
    for s in range(int(z["steps"])):
        g.tt = s * c.dt
        g.step(c.dt, int(z["if_reaction"]), int(z["nsub"]))
    f, di, pr = g.download_state()
    g.close()
    di, pr = interior(di), interior(pr)
    if name in GOLDEN_EXACT:
        assert np.array_equal(f, z["f"]) and np.array_equal(di, z["di"]) and np.array_equal(pr, z["prims"])
    else:
        for m in range(5):
            assert rel_linf(z["f"][m], f[m]) <= TOL
        for m in range(di.shape[0]):
            assert rel_linf(z["di"][m], di[m]) <= TOL
        assert rel_linf(z["prims"][4], pr[4]) <= TOL


# ---------------------------------------------------------------- C3 at its configured size
def test_chem_batch_full_size(oracle, gpu):
    """The 2^20-reactor batch (T 900-2200 K, equivalence ratio 0.3-3, dt log-uniform in 1e-8 to
    1e-6 s, uneven sub-step counts) against the oracle's implicit integrator, every reactor."""
    names, th, kin, di, E, dt, nsub, T = cases.reactors(n=1 << 20, seed=0)
    dio, eo = di.copy(), E.copy()
    oracle.chem_batch(th, kin, 1, abi.CHEM_IMPLICIT, dio, eo, dt, nsub, threads=os.cpu_count() or 1)
    gpu.chem_setup(th, kin, 1, abi.CHEM_IMPLICIT)
    dig, eg = di.copy(), E.copy()
    gpu.chem_batch(dig, eg, dt, nsub)
    scale = np.abs(dio).max(axis=1, keepdims=True)
    err = np.abs(dig - dio) / scale
    assert err.max() <= TOL, err.max()
    assert np.abs(eg - eo).max() <= TOL * np.abs(eo).max()
    assert np.abs(dig - di).max() > 0


def test_chem_batch_constant_pressure(oracle, gpu):
    """C3's constant-pressure reactors (an extension of the reference's constant-volume reactor):
    the GPU applies the oracle's pressure-restoring rule after every sub-step; the reactors keep
    their initial pressure and specific total enthalpy."""
    names, th, kin, di, E, dt, nsub, T = cases.reactors(n=8192, seed=4)
    dio, eo = di.copy(), E.copy()
    oracle.chem_batch(th, kin, 1, abi.CHEM_IMPLICIT, dio, eo, dt, nsub, threads=os.cpu_count() or 1, const_p=True)
    gpu.chem_setup(th, kin, 1, abi.CHEM_IMPLICIT, const_p=True)
    assert gpu.lib().ocfd_gpu_chem_constant_pressure(-1) == 1
    dig, eg = di.copy(), E.copy()
    gpu.chem_batch(dig, eg, dt, nsub)
    gpu.chem_setup(th, kin, 1, abi.CHEM_IMPLICIT)  # back to the reference's reactor
    assert gpu.lib().ocfd_gpu_chem_constant_pressure(-1) == 0
    scale = np.abs(dio).max(axis=1, keepdims=True)
    assert (np.abs(dig - dio) / scale).max() <= TOL
    assert np.abs(eg - eo).max() <= TOL * np.abs(eo).max()
    # pressure held: p = sum R_k d_k T before and after, for a sample of reactors
    for r in range(0, 8192, 512):
        T0 = oracle.probe(th, 1, 1, di[r], E[r])
        T1 = oracle.probe(th, 1, 1, dig[r], eg[r])
        p0, p1 = oracle.probe(th, 1, 2, di[r], T0), oracle.probe(th, 1, 2, dig[r], T1)
        assert abs(p1 - p0) <= 1e-10 * p0
    assert np.abs(dig.sum(axis=1) - di.sum(axis=1)).max() > 0  # the density moved to hold p


def test_cooperative_batch_equals_cell_kernel(gpu):
    """The batched implicit chemistry (warp-cooperative kernel: one lane per species) against the
    flow solver's one-thread-per-cell kernel on the same reacting jet cells: the same operations in
    the same order, so the densities and energies agree bit for bit."""
    c = cases.jet(nx=24, ny=16, nz=16)
    g = gpu.Solver(c)
    g.init_state()
    for s in range(3):
        g.tt = s * c.dt
        g.step(c.dt, 1, c.nsub)
    _, di0, pr0 = g.download_state()
    g.chemical_time_advance(c.dt, 1)
    _, di1, pr1 = g.download_state()
    g.close()
    ns = c.params.n_spec
    D = np.ascontiguousarray(interior(di0).reshape(ns, -1).T)
    E = np.ascontiguousarray(interior(pr0[6]).reshape(-1))
    gpu.chem_setup(c.thermo, c.kin, 1, abi.CHEM_IMPLICIT)
    gpu.chem_batch(D, E, np.full(len(E), c.dt), np.ones(len(E), np.int32))
    assert np.array_equal(D, interior(di1).reshape(ns, -1).T)
    assert np.array_equal(E, interior(pr1[6]).reshape(-1))
    assert np.abs(D - interior(di0).reshape(ns, -1).T).max() > 0
