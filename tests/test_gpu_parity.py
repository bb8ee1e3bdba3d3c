"""Parity of the CUDA hot path (through the C ABI) with the CPU oracle on the same seeded inputs.

Cases whose arithmetic has no transcendental function (perfect or NASA-fit gas, Sutherland /
Pr / Sc transport, every reconstruction, both splittings, CD6 / CD8, boundary-layer and periodic
boundary conditions, ghost cells, Et repair) must agree BIT FOR BIT: the library is built with
--fmad=false and keeps the reference's evaluation order. Cases with exp / log / pow (Wilke
transport, finite-rate chemistry) differ only by the last-place differences of CUDA's and glibc's
libm, and must agree to a relative L-infinity of 1e-10 (the tolerance of the hot path's
correctness target) after several steps.
"""
import numpy as np
import pytest

from ocfd_b200 import abi, cases

pytestmark = pytest.mark.gpu
L = 4


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


def run_pair(oracle, gpu, case, nsteps, if_reaction=0, nsub=1, graph=True):
    o = oracle.OracleSolver(case)
    o.init_state()
    g = gpu.Solver(case)
    g.init_state()
    for s in range(nsteps):
        tt = s * case.dt
        o.step(case.dt, tt, if_reaction, nsub)
        if graph:
            g.tt = tt
            g.step(case.dt, if_reaction, nsub)
        else:
            g.flow_time_advance(0.5 * case.dt, tt)
            if if_reaction:
                g.chemical_time_advance(case.dt / nsub, nsub)
            g.flow_time_advance(0.5 * case.dt, tt)
    so, sg = o.download_state(), g.download_state()
    ro = o.rhybrid() if case.params.scheme_invis == abi.SCHEME_HYBRID else None
    rg = g.rhybrid() if case.params.scheme_invis == abi.SCHEME_HYBRID else None
    do, dg = o.diag(), g.show_flow_msg()
    o.close()
    g.close()
    return so, sg, ro, rg, do, dg


def assert_bitwise(so, sg):
    fo, dio, pro = so
    fg, dig, prg = sg
    assert np.array_equal(fo, fg), [rel_linf(fo[m], fg[m]) for m in range(5)]
    assert np.array_equal(interior(pro), interior(prg)), [rel_linf(pro[m], prg[m]) for m in range(7)]
    assert np.array_equal(interior(dio), interior(dig))


@pytest.mark.parametrize("scheme", ["WENO5", "WENO7", "OMP6", "UD7L"])
def test_isotropic_schemes_bitwise(oracle, gpu, scheme):
    c = cases.isotropic(n=16, scheme=scheme)
    if scheme == "UD7L":
        c.params.ud7l_diss = 0.5
    so, sg, _, _, do, dg = run_pair(oracle, gpu, c, 3)
    assert_bitwise(so, sg)
    assert abs(do[0] - dg[0]) <= 1e-12 * abs(do[0]) and abs(do[1] - dg[1]) <= 1e-12 * abs(do[1])


def test_isotropic_llf_cd8_bitwise(oracle, gpu):
    c = cases.isotropic(n=16, flux_splitting=abi.SPLIT_LLF)
    c.params.scheme_vis = abi.SCHEME_CD8
    so, sg, *_ = run_pair(oracle, gpu, c, 2)
    assert_bitwise(so, sg)


def test_graph_equals_plain_launches(oracle, gpu):
    c = cases.isotropic(n=16)
    so, sg, *_ = run_pair(oracle, gpu, c, 2, graph=False)
    assert_bitwise(so, sg)


@pytest.mark.parametrize("scheme", ["HYBRID", "OMP6", "WENO5"])
def test_flatplate_bitwise(oracle, gpu, scheme):
    c = cases.flatplate(nx=40, ny=24, nz=12, scheme=scheme, lx=0.01, ly=0.004, y1=2e-5)
    so, sg, ro, rg, *_ = run_pair(oracle, gpu, c, 3)
    assert_bitwise(so, sg)
    if ro is not None:
        assert np.array_equal(ro, rg)  # identical hybrid decision inputs
        th1, th2 = c.params.hybrid_para[1], c.params.hybrid_para[2]
        sel = np.digitize(interior(rg), [th1, th2], right=True)
        assert len(np.unique(sel)) >= 2  # the case exercises more than one scheme


def _variant(p, name):
    if name in ("sb_iplus_weno5", "all"):
        p.scheme_boundary[1] = 1   # i+: full WENO5 at the closure interfaces (ghost-cell type)
    if name in ("sb_jplus_none", "all"):
        p.scheme_boundary[3] = -1  # j+: interior scheme up to the face
    if name in ("outlet2", "all"):
        p.bc_para[3] = 2           # second-order outlet extrapolation


@pytest.mark.parametrize("name", ["sb_iplus_weno5", "sb_jplus_none", "outlet2", "all"])
def test_flatplate_boundary_variants_bitwise(oracle, gpu, name):
    """Scheme_boundary = 1 / -1 faces (their closures read the halo, whose metrics are the
    reference's unfilled 1.0) and the second-order outlet."""
    c = cases.flatplate(nx=40, ny=24, nz=12, scheme="WENO5", lx=0.01, ly=0.004, y1=2e-5)
    _variant(c.params, name)
    so, sg, *_ = run_pair(oracle, gpu, c, 2)
    assert_bitwise(so, sg)


def test_general_metrics_bitwise(oracle, gpu):
    """A curvilinear (non tensor-product) grid runs the full 19-array metric path."""
    c = cases.isotropic(n=12)
    X, Y, Z = c.coords
    sl = (slice(L, -L), slice(L, -L), slice(L, -L))
    h = c.info["h"]
    Xi = X[sl].copy()
    X[sl] = Xi + 0.08 * h * np.sin(2 * np.pi * Y[sl] / (12 * h)) * np.cos(2 * np.pi * Z[sl] / (12 * h))
    o = oracle.OracleSolver(c)
    mo = o.metrics()
    o.close()
    g = gpu.Solver(c)
    mg = g.metrics()
    g.close()
    assert np.array_equal(interior(mo), interior(mg))
    so, sg, *_ = run_pair(oracle, gpu, c, 2)
    assert_bitwise(so, sg)


def test_separable_metrics_match_oracle(oracle, gpu):
    c = cases.flatplate(nx=40, ny=24, nz=12, scheme="WENO5", lx=0.01, ly=0.004, y1=2e-5)
    o = oracle.OracleSolver(c)
    mo = o.metrics()
    o.close()
    g = gpu.Solver(c)
    mg = g.metrics()
    assert gpu.lib().ocfd_gpu_is_separable() == 1
    g.close()
    assert np.array_equal(interior(mo), interior(mg))


@pytest.mark.parametrize("kind", ["flatplate", "jet"])
def test_multistep_run_equals_single_steps(gpu, kind):
    """ocfd_gpu_run (chunks of 16 steps per graph launch plus single steps, the wall-disturbance
    time taken on the device) gives the same state as one ocfd_gpu_step per step."""
    if kind == "flatplate":
        c = cases.flatplate(nx=40, ny=24, nz=12, scheme="HYBRID", lx=0.01, ly=0.004, y1=2e-5)
        n, reac, nsub = 37, 0, 1
    else:
        c = cases.jet(nx=24, ny=16, nz=16)
        n, reac, nsub = 18, 1, c.nsub
    out = []
    for multi in (False, True):
        g = gpu.Solver(c)
        g.init_state()
        if multi:
            g.run(c.dt, n, reac, nsub)
        else:
            for s in range(n):
                g.step(c.dt, reac, nsub)
        assert abs(g.tt - n * c.dt) < 1e-12 * n * c.dt
        out.append(g.download_state())
        g.close()
    (f0, d0, p0), (f1, d1, p1) = out
    assert np.array_equal(f0, f1)
    assert np.array_equal(interior(p0), interior(p1)) and np.array_equal(interior(d0), interior(d1))


def test_given_metrics_on_a_tensor_grid(gpu):
    """Metrics handed to ocfd_gpu_init (Iflag_Gridtype = 31) on a tensor-product grid take the
    stored-array path and give the separable path's results bit for bit."""
    c = cases.flatplate(nx=40, ny=24, nz=12, scheme="HYBRID", lx=0.01, ly=0.004, y1=2e-5)
    out = []
    for given in (False, True):
        g = gpu.Solver(c)
        m = g.metrics()
        if given:
            g.close()
            g = gpu.Solver(c, metrics=m)
            assert gpu.lib().ocfd_gpu_is_separable() == 0
        g.init_state()
        for s in range(2):
            g.tt = s * c.dt
            g.step(c.dt, 0, 1)
        out.append(g.download_state())
        g.close()
    (f0, d0, p0), (f1, d1, p1) = out
    assert np.array_equal(f0, f1)
    assert np.array_equal(interior(p0), interior(p1)) and np.array_equal(interior(d0), interior(d1))


def test_two_species_realgas_bitwise(oracle, gpu):
    """N_SPEC = 2 (O2/N2): species transport, Newton T(E), Fickian diffusion with enthalpy flux."""
    c = cases.isotropic(n=12, species=["O2", "N2"], Y=[0.233, 0.767])
    so, sg, *_ = run_pair(oracle, gpu, c, 2)
    assert_bitwise(so, sg)


def test_reacting_nine_species(oracle, gpu):
    """9-species H2-air, Wilke transport, implicit chemistry sub-steps inside the Strang step."""
    names, *_ = cases.h2air_structs()
    Y = [1e-6, 0.2, 0.02, 0.1, 1e-5, 1e-6, 1e-7, 1e-7, 0.68]
    c = cases.isotropic(n=12, species=names, Y=Y, wilke=True, T0=1500.0)
    so, sg, *_ = run_pair(oracle, gpu, c, 3, if_reaction=1, nsub=2)
    fo, dio, pro = so
    fg, dig, prg = sg
    tol = 1e-10
    for m in range(5):
        assert rel_linf(fo[m], fg[m]) <= tol, (m, rel_linf(fo[m], fg[m]))
    for m in range(9):
        assert rel_linf(interior(dio[m]), interior(dig[m])) <= tol, (m, rel_linf(interior(dio[m]), interior(dig[m])))
    assert rel_linf(interior(pro[4]), interior(prg[4])) <= tol


@pytest.mark.parametrize("iflag", [0, 1])
def test_reacting_jet(oracle, gpu, iflag):
    """BC_JET inflow (Dirichlet / subsonic switch), zeroth-order outlet, 9 species, Wilke, chemistry."""
    c = cases.jet(nx=24, ny=16, nz=16, iflag_inlet=iflag)
    so, sg, *_ = run_pair(oracle, gpu, c, 2, if_reaction=1, nsub=1)
    fo, dio, pro = so
    fg, dig, prg = sg
    for m in range(5):
        assert rel_linf(fo[m], fg[m]) <= 1e-10, (m, rel_linf(fo[m], fg[m]))
    for m in range(9):
        assert rel_linf(interior(dio[m]), interior(dig[m])) <= 1e-10


@pytest.mark.parametrize("mode", [abi.CHEM_IMPLICIT, abi.CHEM_EULER, abi.CHEM_RK2, abi.CHEM_RK3])
def test_chem_batch(oracle, gpu, mode):
    """Batched 0-D reactors (persistent work queue) against the oracle integrator."""
    names, th, kin, di, E, dt, nsub, T = cases.reactors(n=4096, seed=1)
    if mode != abi.CHEM_IMPLICIT:
        dt = np.minimum(dt, 2e-9)  # explicit integrators need small steps
        nsub = np.ones_like(nsub)
    dio, eo = di.copy(), E.copy()
    oracle.chem_batch(th, kin, 1, mode, dio, eo, dt, nsub)
    gpu.chem_setup(th, kin, 1, mode)
    dig, eg = di.copy(), E.copy()
    gpu.chem_batch(dig, eg, dt, nsub)
    scale = np.abs(dio).max(axis=1, keepdims=True)
    err = np.abs(dig - dio) / scale
    assert err.max() <= 1e-10, err.max()
    assert np.abs(eg - eo).max() <= 1e-10 * np.abs(eo).max()
    assert np.abs(dig - di).max() > 0  # chemistry actually advanced


def test_negative_energy_repair_bitwise(oracle, gpu):
    c = cases.isotropic(n=12)
    o = oracle.OracleSolver(c)
    o.init_state()
    f, di, pr = o.download_state()
    f[4, 5, 6, 7] = 0.25 * (f[1, 5, 6, 7] ** 2) / f[0, 5, 6, 7]
    f[4, 5, 6, 8] = 0.25 * (f[1, 5, 6, 8] ** 2) / f[0, 5, 6, 8]
    o.upload_state(f, di, pr)
    g = gpu.Solver(c)
    g.upload_state(f, di, pr)
    o.flow_time_advance(1e-12, 0.0)
    g.flow_time_advance(1e-12, 0.0)
    assert g.stats()[0] >= 1
    assert_bitwise(o.download_state(), g.download_state())
    # more than ten such cells stop the run, as the reference does
    f[4, 2:6, 2:6, 2:6] = 0.0
    g.upload_state(f, di, pr)
    with pytest.raises(gpu.OcfdError) as ei:
        g.flow_time_advance(1e-12, 0.0)
    assert ei.value.code == abi.ERR_NEGATIVE_ET
    o.close()
    g.close()


def test_bad_parameters_rejected(gpu):
    c = cases.isotropic(n=12)
    c.params.ghost_cell[0] = -1  # user-defined ghost cells
    with pytest.raises(gpu.OcfdError) as ei:
        gpu.Solver(c)
    assert ei.value.code == abi.ERR_UNSUPPORTED
    c = cases.isotropic(n=12)
    c.params.scheme_invis = 7
    with pytest.raises(gpu.OcfdError) as ei:
        gpu.Solver(c)
    assert ei.value.code == abi.ERR_PARAM
    c = cases.isotropic(n=12)
    c.params.ibc = 108  # a boundary-condition family the library does not carry
    with pytest.raises(gpu.OcfdError) as ei:
        gpu.Solver(c)
    assert ei.value.code == abi.ERR_UNSUPPORTED


# ---------------------------------------------------------------- characteristic-space flux
@pytest.mark.parametrize("scheme", ["WENO5", "WENO7", "OMP6"])
def test_characteristic_isotropic_bitwise(oracle, gpu, scheme):
    """IF_Scheme_Character = 1 on a periodic box: projections on the eigenvectors of the
    interface-averaged state, component-wise reconstruction, back projection."""
    c = cases.isotropic(n=16, scheme=scheme)
    c.params.if_scheme_character = 1
    so, sg, *_ = run_pair(oracle, gpu, c, 2)
    assert_bitwise(so, sg)


@pytest.mark.parametrize("variant", ["default", "all"])
def test_characteristic_flatplate_bitwise(oracle, gpu, variant):
    """HYBRID with the characteristic flux: linear interfaces skip the projection, closed faces
    take the boundary closures and the non-reflecting physical flux at interfaces 0 and n."""
    c = cases.flatplate(nx=40, ny=24, nz=12, scheme="HYBRID", lx=0.01, ly=0.004, y1=2e-5)
    c.params.if_scheme_character = 1
    if variant == "all":
        _variant(c.params, "all")
    so, sg, *_ = run_pair(oracle, gpu, c, 2)
    assert_bitwise(so, sg)


def test_characteristic_llf_weno5_flatplate_bitwise(oracle, gpu):
    c = cases.flatplate(nx=40, ny=24, nz=12, scheme="WENO5", lx=0.01, ly=0.004, y1=2e-5)
    c.params.if_scheme_character = 1
    c.params.flux_splitting = abi.SPLIT_LLF
    so, sg, *_ = run_pair(oracle, gpu, c, 2)
    assert_bitwise(so, sg)


# ---------------------------------------------------------------- ghost cells
GHOST_CASES = {
    "wall_copy_weno5": {2: (1, 1)},                 # j- wall: Ghost_Cell 1, Scheme_boundary 1
    "outlet_mirror_inner": {1: (2, -1)},            # i+ outlet: Ghost_Cell 2, Scheme_boundary -1
    "upper_mirror_weno5": {3: (2, 1)},              # j+ upper: Ghost_Cell 2, Scheme_boundary 1
    "three_faces": {1: (2, 1), 2: (1, 1), 3: (2, -1)},
}


@pytest.mark.parametrize("name", list(GHOST_CASES))
def test_ghost_cells_flatplate_bitwise(oracle, gpu, name):
    """Ghost_Cell 1 / 2 faces: the Jacobian ghost slabs of init_mesh (copy or mirrored
    coordinates + comput_Jacobian3d_Ghost) and the flow extrapolation after every boundary
    condition, read by the WENO5 (Scheme_boundary 1) or interior (-1) schemes at the face."""
    c = cases.flatplate(nx=40, ny=24, nz=12, scheme="WENO5", lx=0.01, ly=0.004, y1=2e-5)
    for face, (gc, sb) in GHOST_CASES[name].items():
        c.params.ghost_cell[face] = gc
        c.params.scheme_boundary[face] = sb
    o = oracle.OracleSolver(c)
    mo = o.metrics()
    o.close()
    g = gpu.Solver(c)
    mg = g.metrics()
    g.close()
    assert np.array_equal(mo, mg)  # full halo arrays, ghost slabs included
    so, sg, *_ = run_pair(oracle, gpu, c, 2)
    assert_bitwise(so, sg)
    pro, prg = so[2], sg[2]
    for face in GHOST_CASES[name]:  # the ghost cells of the primitive arrays too
        dim = 3 - face // 2  # arrays are (var, k, j, i)
        sl = [slice(None), slice(L, -L), slice(L, -L), slice(L, -L)]
        sl[dim] = slice(0, L) if face % 2 == 0 else slice(-L, None)
        assert np.array_equal(pro[tuple(sl)], prg[tuple(sl)])
