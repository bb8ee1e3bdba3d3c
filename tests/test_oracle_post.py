"""Oracle restatement of filtering (code/others/OCFD_filtering.f90) and of the analysis routines
(code/others/OCFD_ANA.f90) on the CPU: properties of the filters that follow from their
coefficients, the box and boundary rules, and the isotropic-turbulence statistics of the 64^3
start state (the workload's M_t = 0.3, Re_lambda ~ 70 construction)."""
import numpy as np
import pytest

from ocfd_b200 import cases, post


def _solver(oracle, c, steps=1):
    o = oracle.OracleSolver(c)
    o.init_state()
    for s in range(steps):
        o.step(c.dt, s * c.dt, 0, 1)
    return o


def test_fo9p_coefficients_remove_the_grid_mode_and_keep_constants(oracle):
    """Transfer function of the 9-point filter: 0 at k = 0, 1 at k = pi (s0 = 1)."""
    c = cases.isotropic(n=16)
    o = _solver(oracle, c)
    f, di, prims = o.download_state()
    nx = c.shape[0]
    i = np.arange(nx)
    base = f.copy()
    base[:] = base.mean(axis=(1, 2, 3), keepdims=True)  # uniform in every component
    g = base.copy()
    g[0] += 1e-3 * base[0] * ((-1.0) ** i)[None, None, :]  # odd-even mode in x on the density
    o.upload_state(np.ascontiguousarray(g), di, prims)
    t, n = post.filter_table([dict(step=1, x=1, scheme=post.FILTER_FO9P, s0=1.0)])
    assert o.filtering(1, t, n) == 1
    f1, _, _ = o.download_state()
    assert np.abs(f1 - base).max() <= 1e-12 * np.abs(base).max()
    o.close()


def test_filter_cadence_box_and_walls(oracle):
    c = cases.flatplate(nx=40, ny=24, nz=12, scheme="WENO5", lx=0.01, ly=0.004, y1=2e-5)
    o = _solver(oracle, c)
    f0, _, _ = o.download_state()
    t, n = post.filter_table([dict(step=3, y=1, scheme=post.FILTER_FO9P, s0=0.5, box=((10, 30), (1, 1000), (2, 7))),
                              dict(step=2, x=1, scheme=post.FILTER_FO9P, s0=0.5, box=((1, 1000), (3, 3), (1, 1)))])
    assert o.filtering(5, t, n) == 0  # neither group is due
    assert np.array_equal(o.download_state()[0], f0)
    assert o.filtering(3, t, n) == 1  # the y group
    f1, di, prims = o.download_state()
    kk, jj, ii = np.nonzero(np.abs(f1 - f0).max(axis=0))  # (nz, ny, nx), 0-based
    assert ii.min() == 9 and ii.max() == 29  # x box 10..30
    assert kk.min() == 1 and kk.max() == 6   # z box 2..7
    assert jj.min() == 5 and jj.max() == 24 - 6  # y is not periodic: j = 6 .. ny-5
    o.upload_state(f0, di, prims)
    assert o.filtering(2, t, n) == 1  # the x group: one line
    f2, _, _ = o.download_state()
    kk, jj, ii = np.nonzero(np.abs(f2 - f0).max(axis=0))
    assert set(kk) == {0} and set(jj) == {2}
    assert ii.min() == 5 and ii.max() == 40 - 6  # x is not periodic either
    o.close()


def test_shock_filter_acts_only_where_pressure_jumps(oracle):
    c = cases.isotropic(n=16)
    o = _solver(oracle, c)
    f0, di, prims = o.download_state()
    # rth = 0 gives sc0 = 1 everywhere (100 % filtering); a huge rth gives sc0 = 0 (no filtering)
    t, n = post.filter_table([dict(step=1, z=1, scheme=post.FILTER_SHOCK, s0=1.0, rth=1e30)])
    o.filtering(1, t, n)
    f1, _, _ = o.download_state()
    assert np.array_equal(f0, f1)
    o.upload_state(f0, di, prims)
    t, n = post.filter_table([dict(step=1, z=1, scheme=post.FILTER_SHOCK, s0=1.0, rth=0.0)])
    o.filtering(1, t, n)
    f2, _, _ = o.download_state()
    assert np.abs(f2 - f0).max() > 0
    # conservative form: the periodic sum of each variable is kept to rounding
    scale = np.abs(f0).sum(axis=(1, 2, 3))
    assert (np.abs(f2.sum(axis=(1, 2, 3)) - f0.sum(axis=(1, 2, 3))) <= 1e-12 * scale).all()
    o.close()


def test_ana_box_of_the_isotropic_start_state(oracle):
    """The 64^3 start state is built for M_t = 0.3 and Re_lambda ~ 70 with ana_box's definitions."""
    c = cases.isotropic(n=64)
    o = _solver(oracle, c, steps=1)  # comput_Amu_Amk_AMD has run
    row = dict(zip(post.BOX_COLUMNS, o.ana_box(c.dt)))
    assert row["tt"] == c.dt
    assert abs(row["Amt"] - 0.3) < 0.02, row
    assert 50 < row["Re_lamda"] < 90, row
    assert abs(row["u_skewness"]) < 0.3 and 2.0 < row["u_flatness"] < 4.0, row
    assert row["ux_skewness"] < 0.0, row  # velocity-derivative skewness of decaying turbulence
    o.close()


def test_time_average_of_a_constant_state_is_the_state(oracle):
    c = cases.isotropic(n=8)
    o = _solver(oracle, c, steps=0)
    for m in range(3):
        k, t = o.ana_time_average(c.dt)
    assert k == 3 and abs(t - 3 * c.dt) < 1e-18
    a = o.ana_average()
    f, di, prims = o.download_state()
    L = 4
    assert np.allclose(a[0], prims[0][L:-L, L:-L, L:-L], rtol=1e-15, atol=0)
    assert np.allclose(a[4], prims[4][L:-L, L:-L, L:-L], rtol=1e-15, atol=0)
    o.close()


def test_q_of_solid_rotation(oracle):
    """Q = Omega^2 for u = -Omega y, v = Omega x (a vortex core); the central scheme is exact for
    linear fields away from the boundary closures, which are also exact for linear fields."""
    c = cases.flatplate(nx=16, ny=16, nz=8, scheme="WENO5", lx=0.01, ly=0.004, y1=2e-5)
    o = _solver(oracle, c, steps=0)
    f, di, prims = o.download_state()
    X, Y = c.coords[0], c.coords[1]
    om = 50.0
    prims = prims.copy()
    prims[1] = -om * Y
    prims[2] = om * X
    o.upload_state(f, di, prims)
    q = o.ana_q()
    L = 4
    assert np.allclose(q[:, 2:-2, 2:-2], om * om, rtol=1e-6), (q.min(), q.max())
    o.close()
