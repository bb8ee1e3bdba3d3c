"""The compiled host driver (opencfd-comb_b200/host/ns_solver.cpp): NS_solver's call sequence
(code/flow-solver/OCFD_NS_Solver.f90:9-70) replayed over the C ABI from a case file. On the CPU the
case file written by Case.save is read back by the driver (--describe); on the GPU the driver's
final state equals, bit for bit, the same call sequence made from Python."""
import os
import subprocess

import numpy as np
import pytest

from ocfd_b200 import cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "opencfd-comb_b200", "host", "ocfd_ns_solver")


def _need_exe():
    if not os.path.exists(EXE):
        pytest.skip("host driver not built (make -C opencfd-comb_b200)")


def _fields(out):
    kv = dict(tok.split("=") for tok in out.split())
    return {k: (float(v) if any(ch in v for ch in ".e") else int(v)) for k, v in kv.items()}


@pytest.mark.parametrize("make", ["jet", "flatplate"])
def test_case_file_roundtrip(tmp_path, make):
    _need_exe()
    if make == "jet":
        c = cases.jet(nx=24, ny=16, nz=16, nsteps=3)
    else:
        c = cases.flatplate(nx=40, ny=24, nz=12, scheme="WENO5", lx=0.01, ly=0.004, y1=2e-5, nsteps=3)
    path = tmp_path / "case.bin"
    c.save(str(path))
    r = subprocess.run([EXE, "--describe", str(path)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    d = _fields(r.stdout)
    nx, ny, nz = c.shape
    assert (d["nx"], d["ny"], d["nz"], d["lap"]) == (nx, ny, nz, 4)
    assert d["n_spec"] == c.params.n_spec
    assert (d["nsteps"], d["if_reaction"], d["nsub"]) == (c.nsteps, c.if_reaction, c.nsub)
    assert d["dt"] == c.dt
    assert d["kinetics"] == (1 if c.kin is not None else 0)
    assert d["bc"] == (1 if c.bc is not None else 0)
    # sums of what the driver read (accumulation order differs from numpy's: relative 1e-9)
    assert abs(d["sum_coords"] - float(np.sum(c.coords))) <= 1e-9 * max(1.0, abs(float(np.sum(c.coords))))
    assert abs(d["sum_prim"] - float(np.sum(c.prim5))) <= 1e-9 * abs(float(np.sum(c.prim5)))
    assert abs(d["sum_di"] - float(np.sum(c.di))) <= 1e-9 * max(1.0, abs(float(np.sum(c.di))))


def test_truncated_case_file_is_an_error(tmp_path):
    _need_exe()
    c = cases.isotropic(n=8)
    path = tmp_path / "case.bin"
    c.save(str(path))
    data = path.read_bytes()
    path.write_bytes(data[:len(data) // 2])
    r = subprocess.run([EXE, "--describe", str(path)], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0
    assert "truncated" in r.stderr


def _python_run(c):
    """The same sequence from Python: flow(dt/2), chemistry x nsub, flow(dt/2), show_flow_msg."""
    from ocfd_b200 import solver
    g = solver.Solver(c)
    g.init_state()
    tt, msgs = 0.0, []
    show = c.params.istep_show if c.params.istep_show > 0 else 1
    for istep in range(1, c.nsteps + 1):
        g.flow_time_advance(0.5 * c.dt, tt)
        if c.if_reaction:
            g.chemical_time_advance(c.dt / c.nsub, c.nsub)
        g.flow_time_advance(0.5 * c.dt, tt)
        tt = tt + c.dt
        if istep % show == 0:
            msgs.append(g.show_flow_msg())
    st = g.download_state()
    g.close()
    return st, msgs


@pytest.mark.gpu
@pytest.mark.parametrize("make", ["jet", "flatplate"])
def test_host_driver_matches_python_driver(tmp_path, make):
    _need_exe()
    if make == "jet":
        c = cases.jet(nx=24, ny=16, nz=16, nsteps=3)
    else:
        c = cases.flatplate(nx=40, ny=24, nz=12, scheme="HYBRID", lx=0.01, ly=0.004, y1=2e-5, nsteps=3)
    path, out = tmp_path / "case.bin", tmp_path / "state.bin"
    c.save(str(path))
    r = subprocess.run([EXE, str(path), str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    (f, di, prims), msgs = _python_run(c)
    raw = np.fromfile(str(out), dtype=np.float64)
    assert raw.size == f.size + di.size + prims.size
    f1 = raw[:f.size].reshape(f.shape)
    di1 = raw[f.size:f.size + di.size].reshape(di.shape)
    p1 = raw[f.size + di.size:].reshape(prims.shape)
    assert np.array_equal(f, f1)
    assert np.array_equal(di, di1)
    assert np.array_equal(prims, p1)
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("Istep=")]
    assert len(lines) == len(msgs)
    for ln, (e, k) in zip(lines, msgs):
        d = _fields(ln)
        assert float("%.15e" % e) == d["E_mean"] and float("%.15e" % k) == d["K_mean"]


@pytest.mark.gpu
def test_host_driver_filtering_and_analysis(tmp_path):
    """NS_solver's filtering (:48) and OCFD_analysis (:55) calls from the compiled driver: the
    final state equals the Python sequence with the same calls, and the statistics rows and the
    Q / average files match what post.analysis writes for that sequence."""
    import filecmp
    from ocfd_b200 import post, solver
    _need_exe()
    c = cases.isotropic(n=16)
    c.nsteps = 4
    c.filters = [dict(step=2, x=1, y=1, z=1, scheme=post.FILTER_FO9P, s0=0.3),
                 dict(step=3, z=1, scheme=post.FILTER_SHOCK, s0=1.0, rth=1e-6)]
    c.analysis = [(post.ANA_BOX, 1), (post.ANA_Q, 4), (post.ANA_TIME_AVERAGE, 1, [2])]
    run_dir, py_dir = tmp_path / "c", tmp_path / "py"
    run_dir.mkdir(); py_dir.mkdir()
    c.save(str(run_dir / "case.bin"))
    r = subprocess.run([EXE, "case.bin", "state.bin"], capture_output=True, text=True, timeout=600, cwd=str(run_dir))
    assert r.returncode == 0, r.stderr
    ft, nf = post.filter_table(c.filters)
    at, na = post.ana_table(c.analysis)
    g = solver.Solver(c)
    g.init_state()
    g.keep_viscosity(True)
    tt = 0.0
    for istep in range(1, c.nsteps + 1):
        g.flow_time_advance(0.5 * c.dt, tt)
        g.flow_time_advance(0.5 * c.dt, tt)
        tt = tt + c.dt
        g.filtering(istep, ft, nf)
        post.analysis(g, istep, tt, at, na, outdir=str(py_dir))
    f, di, prims = g.download_state()
    g.close()
    raw = np.fromfile(str(run_dir / "state.bin"), dtype=np.float64)
    assert np.array_equal(raw[:f.size].reshape(f.shape), f)
    assert np.array_equal(raw[f.size + di.size:].reshape(prims.shape), prims)
    for name in ("Q-0000004.dat", "OCFD-comb00000002.dat.average", "OCFD-comb00000004.dat.average"):
        assert filecmp.cmp(str(run_dir / name), str(py_dir / name), shallow=False), name
    rows_c = [[float(x) for x in ln.split()] for ln in (run_dir / "statistics.dat").read_text().splitlines()]
    rows_p = [[float(x) for x in ln.split()] for ln in (py_dir / "statistics.dat").read_text().splitlines()]
    assert rows_c == rows_p and len(rows_c) == c.nsteps
