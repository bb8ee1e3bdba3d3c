"""The learned chemistry surrogate: gradients of the library's tensor-core training pass against the
CPU reference of the network, training progress, and the gated surrogate against the FP64 implicit
integrator on held-out reactors (accuracy, exact element conservation, what the trained network
gains over no network)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sg():
    from ocfd_b200 import surrogate
    return surrogate.Surrogate()


def test_gradients_match_cpu_reference(sg):
    import pymlp
    L = sg.L
    assert L.ocfd_gpu_surrogate_init(3) == 0
    nblob = L.ocfd_gpu_surrogate_blob(None, 0, 0)
    blob = (C.c_float * nblob)()
    assert L.ocfd_gpu_surrogate_blob(blob, nblob, 0) == 0
    params = pymlp.unpack(np.frombuffer(blob, dtype=np.float32))
    rng = np.random.default_rng(5)
    B, nout = 256, sg.ns + 1
    x = np.zeros((B, 16), np.float32)
    x[:, :sg.ns + 3] = rng.standard_normal((B, sg.ns + 3))
    t = np.zeros((B, 16), np.float32)
    t[:, :nout] = rng.standard_normal((B, nout))
    g = np.zeros(sum(r * c + r for r, c in zip(pymlp.ROWS, pymlp.COLS)), np.float32)
    loss = C.c_double()
    fp = C.POINTER(C.c_float)
    assert L.ocfd_gpu_surrogate_grad(B, x.ctypes.data_as(fp), t.ctypes.data_as(fp), g.ctypes.data_as(fp),
                                     C.byref(loss)) == 0
    ref_loss, ref = pymlp.loss_and_grads(params, x.astype(np.float64), t.astype(np.float64), nout)
    # the GPU's GELU uses the hardware tanh (absolute error about 5e-4 on tanh), the reference the
    # exact one: a few BF16 activations round the other way, so the loss agrees to about 1e-5
    assert abs(loss.value - ref_loss) <= 1e-4 * ref_loss
    p = 0
    for l, (r, c) in enumerate(zip(pymlp.ROWS, pymlp.COLS)):
        gw = g[p:p + r * c].reshape(r, c)
        p += r * c
        gb = g[p:p + r]
        p += r
        rw, rb = ref[l]
        assert np.abs(gw - rw).max() <= 5e-3 * np.abs(rw).max(), l
        assert np.abs(gb - rb).max() <= 5e-3 * np.abs(rb).max(), l


@pytest.fixture(scope="module")
def trained(sg):
    hist = sg.train(n=1 << 17, epochs=12, batch=1024, lr=2e-3, seed=0)
    return sg, hist


def test_training_reduces_loss(trained):
    sg, hist = trained
    assert np.isfinite(hist).all()
    assert hist[-1] < 0.2 * hist[0], hist


def test_gated_surrogate_against_fp64(trained):
    sg, _ = trained
    tol_T = 5.0
    r = sg.evaluate(n=1 << 15, seed=4242, tol_T=tol_T)
    # element (and so total) mass conserved to rounding by the projection
    assert r["element_residual_max"] <= 1e-12, r
    # accepted reactors are within the gate, the rest took the FP64 path
    assert r["fallback_fraction"] < 1.0, r
    assert r["gated_T_err_rel_max"] <= 0.01, r
    assert r["gated_Y_err_max"] <= 1e-2, r
    # the trained network gains over no network: far smaller errors than assuming no reaction
    assert r["ungated_T_err_max_K"] < 0.5 * r["no_reaction_T_err_max_K"], r


def test_fused_network_equals_layer_gemms(trained):
    """The fused four-layer kernel and the per-layer GEMMs issue the same MMAs and epilogue
    arithmetic: identical network outputs, so identical gated results."""
    sg, _ = trained
    t = sg.torch
    n = 3 * 128 + 37  # ragged last tile
    di, E, dt, nsub = sg.reactors(n, seed=77)
    outs = []
    for fused in (0, 1):
        was = sg.L.ocfd_gpu_surrogate_fused(fused)
        d_di, d_e, d_dt = [t.from_numpy(np.ascontiguousarray(a)).to("cuda") for a in (di, E, dt)]
        o_di, o_e = t.empty_like(d_di), t.empty_like(d_e)
        Tp, Te = t.empty_like(d_e), t.empty_like(d_e)
        t.cuda.synchronize()
        assert sg.L.ocfd_gpu_surrogate_predict(n, d_di.data_ptr(), d_e.data_ptr(), d_dt.data_ptr(), o_di.data_ptr(),
                                               o_e.data_ptr(), Tp.data_ptr(), Te.data_ptr()) == 0
        outs.append([x.cpu().numpy() for x in (o_di, o_e, Tp, Te)])
        sg.L.ocfd_gpu_surrogate_fused(was)
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


def test_blob_roundtrip(trained):
    sg, _ = trained
    b = sg.blob()
    sg.load(b)
    assert np.array_equal(sg.blob(), b)


def _jet_run(sg, mode, tol, steps=2):
    from ocfd_b200 import cases, solver
    c = cases.jet(nx=24, ny=16, nz=16)
    g = solver.Solver(c)
    g.init_state()
    if mode:
        assert sg.L.ocfd_gpu_chem_mode(1, tol) == 0
    for s in range(steps):
        g.tt = s * c.dt
        g.step(c.dt, 1, c.nsub)
    st = g.download_state()
    rej = sg.L.ocfd_gpu_chem_surrogate_rejected(None) if mode else 0
    g.close()
    return st, rej


def test_flow_surrogate_rejecting_every_cell_is_the_fp64_path(trained):
    """With a gate that accepts nothing, every cell takes the FP64 sub-steps of the list kernel,
    which must reproduce the plain chemistry of the Strang step bit for bit."""
    sg, _ = trained
    (f0, di0, p0), _ = _jet_run(sg, 0, 1.0)
    (f1, di1, p1), rej = _jet_run(sg, 1, 1e-300)
    assert rej == 24 * 16 * 16
    L = 4
    assert np.array_equal(f0, f1)
    assert np.array_equal(di0[:, L:-L, L:-L, L:-L], di1[:, L:-L, L:-L, L:-L])
    assert np.array_equal(p0[:, L:-L, L:-L, L:-L], p1[:, L:-L, L:-L, L:-L])


def test_flow_surrogate_close_to_fp64(trained):
    sg, _ = trained
    (f0, di0, p0), _ = _jet_run(sg, 0, 1.0)
    (f1, di1, p1), rej = _jet_run(sg, 1, 5.0)
    L = 4
    T0, T1 = p0[4][L:-L, L:-L, L:-L], p1[4][L:-L, L:-L, L:-L]
    assert np.abs(T1 - T0).max() <= 0.01 * T0.max()
    Y0 = di0[:, L:-L, L:-L, L:-L] / di0[:, L:-L, L:-L, L:-L].sum(axis=0)
    Y1 = di1[:, L:-L, L:-L, L:-L] / di1[:, L:-L, L:-L, L:-L].sum(axis=0)
    assert np.abs(Y1 - Y0).max() <= 1e-3
