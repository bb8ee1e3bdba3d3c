"""Filtering and analysis on the GPU against the oracle: filters bit for bit (no transcendental
function is involved), the steps after a filter bit for bit (the graph re-captures after the
shock filter moves the energy buffer), Q and the time averages bit for bit, and the ana_box
statistics to 1e-12 relative (the sums run in a different order)."""
import numpy as np
import pytest

from ocfd_b200 import cases, post, solver

pytestmark = pytest.mark.gpu

L4 = 4


def _pair(oracle, c, steps=1, keep=False):
    g = solver.Solver(c)
    g.init_state()
    if keep:
        g.keep_viscosity(True)
    o = oracle.OracleSolver(c)
    o.init_state()
    for s in range(steps):
        g.tt = s * c.dt
        g.step(c.dt, c.if_reaction, c.nsub)
        o.step(c.dt, s * c.dt, c.if_reaction, c.nsub)
    return g, o


def _same(g, o):
    """f whole, primitives and species interiors (halo points the steps never read may differ,
    as in every parity test)."""
    (fg, dg, pg), (fo, do, po) = g.download_state(), o.download_state()
    assert np.array_equal(fg, fo)
    inner = (Ellipsis, slice(L4, -L4), slice(L4, -L4), slice(L4, -L4))
    assert np.array_equal(pg[inner], po[inner])
    assert np.array_equal(dg[inner], do[inner])


FILTERS = {
    "fo9p_xyz": [dict(step=1, x=1, y=1, z=1, scheme=post.FILTER_FO9P, s0=0.7)],
    "shock_xyz": [dict(step=1, x=1, y=1, z=1, scheme=post.FILTER_SHOCK, s0=1.0, rth=1e-5)],
    "boxes": [dict(step=2, x=1, scheme=post.FILTER_FO9P, s0=1.0, box=((5, 12), (2, 9), (1, 4))),
              dict(step=1, y=1, z=1, scheme=post.FILTER_SHOCK, s0=0.5, rth=1e-7, box=((1, 999), (3, 10), (2, 11))),
              dict(step=3, z=1, scheme=post.FILTER_FO9P, s0=1.0)],
}


@pytest.mark.parametrize("kind", ["isotropic", "flatplate"])
@pytest.mark.parametrize("filters", sorted(FILTERS))
def test_filtering_bitwise(oracle, kind, filters):
    if kind == "isotropic":
        c = cases.isotropic(n=16)
    else:
        c = cases.flatplate(nx=40, ny=24, nz=12, scheme="HYBRID", lx=0.01, ly=0.004, y1=2e-5)
    g, o = _pair(oracle, c)
    t, n = post.filter_table(FILTERS[filters])
    for istep in (2, 3):  # the reference filters after Istep has advanced
        assert g.filtering(istep, t, n) == o.filtering(istep, t, n)
        _same(g, o)
        g.tt = (istep - 1) * c.dt
        g.step(c.dt, 0, 1)  # the step after a filter: graph replay on the filtered state
        o.step(c.dt, (istep - 1) * c.dt, 0, 1)
        _same(g, o)
    g.close(); o.close()


def test_bad_filter_table_is_rejected():
    c = cases.isotropic(n=8)
    g = solver.Solver(c)
    g.init_state()
    t, n = post.filter_table([dict(step=0, x=1)])
    with pytest.raises(solver.OcfdError):
        g.filtering(1, t, n)
    g.close()


@pytest.mark.parametrize("kind", ["isotropic", "jet"])
def test_ana_box_against_oracle(oracle, kind):
    c = cases.isotropic(n=16) if kind == "isotropic" else cases.jet(nx=24, ny=16, nz=16)
    g, o = _pair(oracle, c, steps=2, keep=(kind == "isotropic"))
    a, b = g.ana_box(2 * c.dt), o.ana_box(2 * c.dt)
    assert a[0] == b[0]
    # the single-species states are bitwise equal, so only the summation order differs; the
    # reacting jet's states agree to the chemistry tolerance. The absolute floor covers
    # skewness-like sums of terms that nearly cancel.
    rel, floor = (1e-12, 1e-14) if kind == "isotropic" else (1e-9, 1e-12)
    assert np.all(np.abs(a - b) <= rel * np.abs(b) + floor), (a, b)
    g.close(); o.close()


def test_ana_box_needs_the_kept_viscosity():
    c = cases.isotropic(n=8)
    g = solver.Solver(c)
    g.init_state()
    with pytest.raises(solver.OcfdError):
        g.ana_box()
    g.close()


def test_ana_q_and_time_average_bitwise(oracle, tmp_path):
    from ocfd_b200 import files
    c = cases.flatplate(nx=40, ny=24, nz=12, scheme="WENO5", lx=0.01, ly=0.004, y1=2e-5)
    g, o = _pair(oracle, c, steps=1)
    assert np.array_equal(g.ana_q(), o.ana_q())
    for s in range(3):
        kg, tg = g.ana_time_average(c.dt)
        ko, to = o.ana_time_average(c.dt)
        assert (kg, tg) == (ko, to)
        g.tt = (s + 1) * c.dt
        g.step(c.dt, 0, 1)
        o.step(c.dt, (s + 1) * c.dt, 0, 1)
    ag, k, t = g.ana_average()
    assert np.array_equal(ag, o.ana_average())
    # restart round trip through the reference's .average file
    p = tmp_path / "a.average"
    files.write_average(str(p), k, t, list(ag))
    k2, t2, a2 = files.read_average(str(p), *c.shape, ag.shape[0])
    g.ana_average(upload=(a2, k2, t2))
    ag2, k3, t3 = g.ana_average()
    assert np.array_equal(ag2, ag) and (k3, t3) == (k, t)
    g.close(); o.close()


def test_analysis_dispatch_writes_reference_files(oracle, tmp_path):
    c = cases.isotropic(n=16)
    g, _o = _pair(oracle, c, steps=1, keep=True)
    _o.close()
    table, n = post.ana_table([(post.ANA_BOX, 1), (post.ANA_Q, 2), (post.ANA_TIME_AVERAGE, 1, [2])])
    r1 = post.analysis(g, 1, c.dt, table, n, outdir=str(tmp_path))
    assert set(r1) == {post.ANA_BOX, post.ANA_TIME_AVERAGE}
    r2 = post.analysis(g, 2, 2 * c.dt, table, n, outdir=str(tmp_path))
    assert set(r2) == {post.ANA_BOX, post.ANA_Q, post.ANA_TIME_AVERAGE}
    assert (tmp_path / "Q-0000002.dat").exists() and (tmp_path / "OCFD-comb00000002.dat.average").exists()
    rows = (tmp_path / "statistics.dat").read_text().splitlines()
    assert len(rows) == 2 and len(rows[0].split()) == 19
    g.close()
