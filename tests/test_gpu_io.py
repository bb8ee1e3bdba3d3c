"""Save and show without a host sync: snapshots packed on the device and copied to
pinned memory on a copy stream while the next steps run equal the state at the snapshot bit for
bit; the asynchronous show_flow_msg equals the synchronous one; save_flow_data_async writes the
reference's OCFD-comb<Istep>.dat layout byte for byte as a synchronous save would."""
import filecmp

import numpy as np
import pytest

from ocfd_b200 import cases, files, solver

pytestmark = pytest.mark.gpu
L4 = 4


def _fields(g):
    f, di, prims = g.download_state()
    inner = (Ellipsis, slice(L4, -L4), slice(L4, -L4), slice(L4, -L4))
    return np.concatenate([prims[:5][inner], di[inner]])


@pytest.mark.parametrize("kind", ["flatplate", "jet"])
def test_snapshot_overlapping_steps(kind):
    c = cases.flatplate(nx=40, ny=24, nz=12, scheme="HYBRID", lx=0.01, ly=0.004, y1=2e-5) if kind == "flatplate" \
        else cases.jet(nx=24, ny=16, nz=16)
    ref = []
    g = solver.Solver(c)
    g.init_state()
    for s in range(4):
        g.tt = s * c.dt
        g.step(c.dt, c.if_reaction, c.nsub)
        ref.append(_fields(g))
    g.close()
    g = solver.Solver(c)
    g.init_state()
    got = []
    for s in range(4):
        g.tt = s * c.dt
        g.step(c.dt, c.if_reaction, c.nsub)
        if s in (0, 1):
            g.snapshot(s + 1, (s + 1) * c.dt)
        if s == 1:
            with pytest.raises(solver.OcfdError):
                g.snapshot(99, 0.0)  # two in flight
        if s == 3:
            for _ in range(2):
                ist, tt, a = g.snapshot_wait()
                got.append((ist, tt, a.copy()))
    assert [x[0] for x in got] == [1, 2]
    for ist, tt, a in got:
        assert tt == ist * c.dt
        assert np.array_equal(a, ref[ist - 1])
    with pytest.raises(solver.OcfdError):
        g.snapshot_wait()  # none in flight
    g.close()


def test_async_show_equals_sync():
    c = cases.isotropic(n=16)
    g = solver.Solver(c)
    g.init_state()
    g.step(c.dt, 0, 1)
    e0, k0 = g.show_flow_msg()
    g.diag_begin()
    g.tt = c.dt
    g.step(c.dt, 0, 1)  # runs while the sums travel; they are of the state at diag_begin
    assert g.diag_end() == (e0, k0)
    g.close()


def test_save_flow_data_async_files(tmp_path):
    c = cases.isotropic(n=16)
    g = solver.Solver(c)
    g.init_state()
    for s in range(5):
        g.tt = s * c.dt
        g.step(c.dt, 0, 1)
        ist = s + 1
        g.save_flow_data_async(str(tmp_path / ("a%d.dat" % ist)), ist, ist * c.dt)
        files.write_flow_data(str(tmp_path / ("s%d.dat" % ist)), ist, ist * c.dt, _fields(g))
    g.flush_saves()
    g.close()
    for ist in range(1, 6):
        assert filecmp.cmp(str(tmp_path / ("a%d.dat" % ist)), str(tmp_path / ("s%d.dat" % ist)), shallow=False)
    k, t, a = files.read_flow_data(str(tmp_path / "a5.dat"), *c.shape, c.params.n_spec)
    assert k == 5 and t == 5 * c.dt and a.shape == (6,) + c.shape[::-1]
