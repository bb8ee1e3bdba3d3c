"""Throughput of the OpenCFD-Comb hot path on B200: Mcell-steps/s of whole reference time steps
(two RK3 flow half-steps, chemistry between them when the workload reacts).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload flatplate|isotropic]
  python bench.py --impl reference ...      (the reference algorithm on the host cores)

Workload (default): the Mach 2.25 flat-plate boundary layer, 1024x160x128 cells, HYBRID
UD7L/WENO7/WENO5 with the pressure sensor, CD6 viscous terms, Steger-Warming splitting,
boundary-layer boundary conditions with the Rai blowing/suction strip, seeded synthetic state.
Multi-GPU runs are independent replicas (one per rank, weak scaling): the single-rank solver has
no exchange step, so no collective is invented; ranks meet only for the timing barrier and the
max-over-ranks reduction.

The device-resident number (value) times K graph-replayed steps with CUDA events on the library
stream; the state (several GB) is far larger than the 126 MB L2, so no flush is needed. e2e times
the same steps through the C ABI with the state uploaded from pinned host memory and the
conserved variables downloaded every step. The roofline object names the kernel class with the
largest share of a step, timed live with per-launch CUDA events.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "opencfd-comb_b200"))

METRIC = "Mcell-steps/s on 1 B200: plain FP64 vs surrogate chemistry at ≤1% T error"
UNIT = "Mcell-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="flatplate", choices=["flatplate", "isotropic", "jet", "reactors", "surrogate"],
                    help="flatplate = the headline configuration; isotropic, jet and reactors are the other "
                         "configurations of the metric (64^3 decaying turbulence, the 384x256x256 reacting H2 jet, "
                         "2^20 batched 0-D reactors)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--sg-train", type=int, default=1 << 21, help="surrogate workload: training reactors")
    ap.add_argument("--sg-epochs", type=int, default=20, help="surrogate workload: training epochs")
    ap.add_argument("--sg-tol", type=float, default=5.0, help="surrogate workload: gate tolerance on T (K)")
    ap.add_argument("--surrogate", action="store_true",
                    help="jet workload: compare FP64 chemistry with the gated surrogate (trains it first)")
    ap.add_argument("--character", action="store_true",
                    help="characteristic-space inviscid flux (IF_Scheme_Character = 1) instead of component-wise")
    ap.add_argument("--tiles", default="auto",
                    help="stencil tiles: 'auto' (timed by the autotuner before the warm-up), 'default', or an "
                         "explicit choice of 8 comma-separated ints (see ocfd_gpu_autotune)")
    ap.add_argument("--profile-region", action="store_true",
                    help="bracket the timed region with cudaProfilerStart/Stop, for ncu --profile-from-start off")
    ap.add_argument("--nz", type=int, default=None,
                    help="cells along z (flat plate: 128 = full; jet: 256 = full), for small profiling runs")
    return ap.parse_args()


def profiler(on, enabled):
    """cudaProfilerStart / Stop around a timed region when --profile-region is given."""
    if not enabled:
        return
    import torch
    rt = torch.cuda.cudart()
    (rt.cudaProfilerStart if on else rt.cudaProfilerStop)()


def make_case(workload, nz=None):
    from ocfd_b200 import cases
    if workload == "isotropic":
        return cases.isotropic(n=64), "isotropic-64^3-WENO5-CD6-SW (decaying turbulence, M_t 0.3, Re_lambda 70)"
    if workload == "jet":
        n = nz or 256
        c = cases.jet(nx=384, ny=256, nz=n)
        return c, "jet-%dx%dx%d-H2air-9sp-19reac-WENO5-CD6-Wilke-implicitChem" % c.shape
    c = cases.flatplate(nx=1024, ny=160, nz=nz or 128, scheme="HYBRID")
    return c, "flatplate-1024x160x%d-M2.25-HYBRID(UD7L/WENO7/WENO5)-CD6-SW-BoundaryLayerBC" % (nz or 128)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    def __init__(self, gpu_index=0):
        self.samples = []
        self.proc = None
        self.idx = gpu_index

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx),
                 "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if len(s) > 2 + k and "Active" in s[2 + k]
                          and "Not" not in s[2 + k]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# algorithmic bytes per cell of one launch of each kernel class (double precision):
#  flux_x : read d,u,v,w,p,Et (6) ; write du (5)                          = 11 doubles
#  flux_y / flux_z : read d,u,v,w,p,Et (6) ; read + write du (10)         = 16 doubles
#  visc_ev: read u,v,w,T,d,di (6) ; write Ev1..Ev3 (12)                   = 18 doubles
#  visc_div: read Ev (12) ; read + write du(2..5) (8)                     = 20 doubles
#  rk_prims: read f,fn,du,di,d (17) ; write f,d,u,v,w,T,p,Et,di (13)      = 30 doubles
#  chem (reacting workloads): read + write di (Ns), Et, f5, read T, p          = 22 doubles (Ns = 9)
ALG_BYTES_PER_CELL = {"flux_x": 88, "flux_y": 128, "flux_z": 128, "visc_ev": 144, "visc_div": 160,
                      "rk_prims": 240, "chem": 176}

# algorithmic FP64 operations per cell of one launch on the flat-plate workload (hand count of the
# kernels' arithmetic; a division or a square root counts as one operation; UD7L interfaces: the
# ~2 % of interfaces that take WENO5 are not counted):
#  split (Steger-Warming + sound speed + separable metric) ~160 per point, (C + 8) / C points per
#  cell (C = 56 for x, 24 for y / z); UD7L 15 per component and sign, 150 per interface,
#  (C + 1) / C interfaces per cell; flux difference 4-6 per component.
#  visc_ev: 12 CD6 derivatives (8 each), metrics 12, chain rule 60, Sutherland + Cp + conductivity
#  ~30, stresses and heat flux 48, Ev 60.  visc_div: 12 CD6 derivatives, sum and Jacobian 16.
ALG_FLOPS_PER_CELL = {"flux_x": 356, "flux_y": 394, "flux_z": 402, "visc_ev": 305, "visc_div": 115}


def main_reference(a):
    """The reference's algorithm on the host cores: the C++ restatement of the Fortran (no
    Fortran compiler exists on this image, so the reference binary itself cannot be built)."""
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    cores = pyoracle.lib().ocfd_cpu_set_threads(os.cpu_count() or 1)
    if a.workload in ("reactors", "surrogate"):  # the reference has only the FP64 integrator
        return reactors_reference(a, pyoracle, cores)
    # size the per-step sample so that warmup + steps take about two minutes
    rate = 0.0
    if a.workload == "flatplate":
        probe, _ = make_case(a.workload, nz=8)
        o = pyoracle.OracleSolver(probe)
        o.init_state()
        t0 = time.perf_counter()
        o.step(probe.dt, 0.0)
        rate = probe.ncell / (time.perf_counter() - t0)
        o.close()
    if a.workload == "flatplate":
        nz = int(max(8, min(128, 120.0 * rate / (1024 * 160 * (a.steps + a.warmup)))))
        c, name = make_case(a.workload, nz=nz)
        sample = "per step: one full time step of a 1024x160x%d slab of the workload (z periodic)" % nz
    elif a.workload == "jet":
        from ocfd_b200 import cases
        c, name = cases.jet(nx=96, ny=64, nz=64), make_case("jet", nz=8)[1].replace("96x64x8", "384x256x256")
        sample = "per step: one reacting time step of the jet on a 96x64x64 grid (same physics)"
    else:
        c, name = make_case(a.workload)
        sample = "per step: one full time step of the 64^3 workload"
    reac, nsub = int(getattr(c, "if_reaction", 0) or 0), int(getattr(c, "nsub", 1) or 1)
    o = pyoracle.OracleSolver(c)
    o.init_state()
    for s in range(a.warmup):
        o.step(c.dt, s * c.dt, reac, nsub)
    t0 = time.perf_counter()
    for s in range(a.steps):
        o.step(c.dt, (a.warmup + s) * c.dt, reac, nsub)
    el = time.perf_counter() - t0
    o.close()
    val = c.ncell * a.steps / el / 1e6
    out = {"metric": METRIC, "value": val, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
           "ms_per_step": el * 1e3 / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64", "data": "synthetic (seeded)", "impl": "reference",
           "config": {"workload": make_case(a.workload, nz=8)[1].replace("x8-", "x128-") if a.workload == "flatplate" else name,
                      "sample_cells": c.ncell},
           "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
           "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


# ---------------------------------------------------------------- batched 0-D reactors (2^20)
RMETRIC = "Mreactor-solves/s on 1 B200: 2^20 H2-air reactors, implicit Euler, uneven sub-steps"
RUNIT = "Mreactor-solves/s"


def reactors_reference(a, pyoracle, cores):
    from ocfd_b200 import abi, cases
    n = 8192
    names, th, kin, di, E, dt, nsub, T = cases.reactors(n=n, seed=1)
    for s in range(a.warmup):
        pyoracle.chem_batch(th, kin, 1, abi.CHEM_IMPLICIT, di.copy(), E.copy(), dt, nsub)
    t0 = time.perf_counter()
    for s in range(a.steps):
        pyoracle.chem_batch(th, kin, 1, abi.CHEM_IMPLICIT, di.copy(), E.copy(), dt, nsub)
    el = time.perf_counter() - t0
    val = n * a.steps / el / 1e6
    out = {"metric": RMETRIC, "value": val, "unit": RUNIT, "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
           "ms_per_step": el * 1e3 / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64", "data": "synthetic (seeded)", "impl": "reference",
           "config": {"workload": "reactors-2^20-H2air-9sp-implicitEuler", "sample_reactors": n},
           "cpu_baseline": {"value": val, "unit": RUNIT, "cores": cores, "kind": "port",
                            "sample": "per step: %d reactors drawn like the 2^20 workload" % n},
           "e2e": {"value": val, "unit": RUNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


def main_reactors(a):
    """2^20 independent constant-volume H2-air reactors through the persistent work-queue kernel
    (ocfd_gpu_chem_batch_device); one step = one pass over all reactors."""
    import numpy as np
    import torch
    from ocfd_b200 import abi, cases, solver
    L = solver.lib()
    import ctypes as C
    n = 2 ** 20
    names, th, kin, di, E, dt, nsub, T = cases.reactors(n=n, seed=0)
    solver.chem_setup(th, kin, 1, abi.CHEM_IMPLICIT)
    dev = torch.device("cuda", 0)
    d_di0, d_e0 = torch.from_numpy(di).to(dev), torch.from_numpy(E).to(dev)
    d_dt, d_ns = torch.from_numpy(dt).to(dev), torch.from_numpy(nsub).to(dev)
    d_di, d_e = d_di0.clone(), d_e0.clone()
    torch.cuda.synchronize()
    # the library launches on its own stream: the restoring copies and the events go there too
    st = torch.cuda.ExternalStream(L.ocfd_gpu_stream())

    def one():
        d_di.copy_(d_di0)
        d_e.copy_(d_e0)
        solver.chem_batch_device(n, d_di.data_ptr(), d_e.data_ptr(), d_dt.data_ptr(), d_ns.data_ptr())

    with torch.cuda.stream(st):
        for s in range(a.warmup):
            one()
        st.synchronize()
        with Clocks(0) as clk:
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(st)
            for s in range(a.steps):
                one()
            ev1.record(st)
            st.synchronize()
    ms = ev0.elapsed_time(ev1)
    value = n * a.steps / (ms * 1e-3) / 1e6
    # e2e: host arrays through ocfd_gpu_chem_batch (copies in and out inside the call)
    e2e = None
    if not a.no_e2e:
        hdi, he = di.copy(), E.copy()
        solver.chem_batch(hdi, he, dt, nsub)
        t0 = time.perf_counter()
        ne = max(1, min(a.steps, 5))
        for s in range(ne):
            hdi[:], he[:] = di, E
            solver.chem_batch(hdi, he, dt, nsub)
        el = time.perf_counter() - t0
        e2e = {"value": n * ne / el / 1e6, "unit": RUNIT, "h2d_bytes_per_step": di.nbytes + E.nbytes + dt.nbytes + nsub.nbytes,
               "d2h_bytes_per_step": di.nbytes + E.nbytes, "timing": "host wall clock around each synchronous call"}
    cpu = None
    if not a.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle
        cores = pyoracle.lib().ocfd_cpu_set_threads(os.cpu_count() or 1)
        m = 8192
        _, _, _, sdi, sE, sdt, sns, _ = cases.reactors(n=m, seed=1)
        t0 = time.perf_counter()
        pyoracle.chem_batch(th, kin, 1, abi.CHEM_IMPLICIT, sdi.copy(), sE.copy(), sdt, sns)
        el = time.perf_counter() - t0
        cpu = {"value": m / el / 1e6, "unit": RUNIT, "cores": cores, "kind": "port",
               "sample": "%d reactors drawn like the 2^20 workload" % m}
    sub = int(nsub.sum())
    out = {"metric": RMETRIC, "value": value, "unit": RUNIT, "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
           "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64", "data": "synthetic (seeded)",
           "config": {"workload": "reactors-2^20-H2air-9sp-implicitEuler", "reactors": n, "substeps_total": sub,
                      "substeps_per_s": sub * a.steps / (ms * 1e-3),
                      "l2": "inputs re-copied from a pristine device copy before each pass"},
           "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": None, "clocks": clk.summary()}
    print(json.dumps(out))
    return 0


# ---------------------------------------------------------------- surrogate chemistry (C4)
SMETRIC = "Mreactor-solves/s on 1 B200: plain FP64 vs gated surrogate chemistry at <=1% T error, 2^20 H2-air reactors"
MLP_FLOPS_PER_SAMPLE = 2 * (16 * 256 + 256 * 256 * 2 + 256 * 16)  # padded forward pass


def main_surrogate(a):
    """Trains the surrogate on FP64-integrated reactors, then times the plain FP64 batch and the
    gated surrogate on 2^20 held-out reactors (device-resident inputs restored before every pass)."""
    import numpy as np
    import torch
    import ctypes as C
    from ocfd_b200 import solver, surrogate
    sg = surrogate.Surrogate()
    L = sg.L
    t0 = time.perf_counter()
    hist = sg.train(n=a.sg_train, epochs=a.sg_epochs, batch=1024, lr=2e-3, seed=0)
    train_s = time.perf_counter() - t0
    n = 1 << 20
    di, E, dt, nsub = sg.reactors(n, 4242)
    dev = torch.device("cuda")
    p_di, p_e = torch.from_numpy(di).to(dev), torch.from_numpy(E).to(dev)
    d_dt, d_ns = torch.from_numpy(dt).to(dev), torch.from_numpy(nsub).to(dev)
    w_di, w_e = p_di.clone(), p_e.clone()
    o_di, o_e = torch.empty_like(p_di), torch.empty_like(p_e)
    Tp, Te = torch.empty_like(p_e), torch.empty_like(p_e)
    torch.cuda.synchronize()
    st = torch.cuda.ExternalStream(L.ocfd_gpu_stream())
    nfb = C.c_int()

    def plain():
        w_di.copy_(p_di)
        w_e.copy_(p_e)
        solver.chem_batch_device(n, w_di.data_ptr(), w_e.data_ptr(), d_dt.data_ptr(), d_ns.data_ptr())

    def gated():
        w_di.copy_(p_di)
        w_e.copy_(p_e)
        solver._chk(L.ocfd_gpu_chem_batch_surrogate(n, w_di.data_ptr(), w_e.data_ptr(), d_dt.data_ptr(),
                                                    d_ns.data_ptr(), a.sg_tol, C.byref(nfb)))

    def network():
        solver._chk(L.ocfd_gpu_surrogate_predict(n, p_di.data_ptr(), p_e.data_ptr(), d_dt.data_ptr(),
                                                 o_di.data_ptr(), o_e.data_ptr(), Tp.data_ptr(), Te.data_ptr()))

    def timed(fn, k):
        with torch.cuda.stream(st):
            for _ in range(a.warmup):
                fn()
            st.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(k):
                fn()
            e1.record(st)
            st.synchronize()
        return e0.elapsed_time(e1) / k

    k = max(1, min(a.steps, 5))
    with Clocks(0) as clk:
        ms_plain = timed(plain, k)
        profiler(True, a.profile_region)
        ms_gated = timed(gated, k)
        profiler(False, a.profile_region)
        ms_net = timed(network, k)
    acc = sg.evaluate(n=n, seed=4242, tol_T=a.sg_tol)
    peaks_file = os.path.join(ROOT, "MEASURED_PEAKS.json")
    bf16_peak = None
    if os.path.exists(peaks_file):
        with open(peaks_file) as fh:
            pk = json.load(fh)
        bf16_peak = pk.get("bf16_tflops")
    # network throughput bound from below by the whole gated pass (features, 4 GEMMs, gate, fallback)
    net_tflops = n * MLP_FLOPS_PER_SAMPLE / (ms_gated * 1e-3) / 1e12
    out = {"metric": SMETRIC, "value": n / (ms_gated * 1e-3) / 1e6, "unit": RUNIT, "n_gpus": 1, "steps": k,
           "warmup": a.warmup, "ms_per_step": ms_gated, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "bf16 network + f64 fallback", "data": "synthetic (seeded)",
           "config": {"workload": "reactors-2^20-H2air-9sp gated surrogate (MLP 12-256-256-256-10, GELU)",
                      "train_reactors": a.sg_train, "epochs": a.sg_epochs, "train_seconds": train_s,
                      "loss_first_last": [float(hist[0]), float(hist[-1])], "tol_T_K": a.sg_tol},
           "plain_fp64": {"value": n / (ms_plain * 1e-3) / 1e6, "ms": ms_plain},
           "speedup_vs_plain": ms_plain / ms_gated,
           "accuracy": acc, "fallback_fraction": nfb.value / n,
           "roofline": {"bound": "tensor", "kernel": "gated pass (features, 4 tcgen05 GEMMs, gate, fallback)",
                        "achieved": net_tflops, "peak": bf16_peak, "unit": "TFLOP/s",
                        "frac": (net_tflops / bf16_peak) if bf16_peak else None, "traffic": None,
                        "flops_per_sample": MLP_FLOPS_PER_SAMPLE, "ms": ms_gated,
                        "ungated_predict_ms": ms_net},
           "cpu_baseline": None, "e2e": None, "gpu_launches": None, "clocks": clk.summary()}
    print(json.dumps(out))
    return 0


def main_jet_surrogate(a):
    """C5 with the gated surrogate: the surrogate is trained on 2^21 batch reactors plus cells of a
    jet snapshot, then the jet runs K steps with FP64 chemistry and K steps with the surrogate from
    the same start; the line reports both throughputs and the surrogate run's temperature and
    species errors against the FP64 run."""
    import numpy as np
    import ctypes as C
    from ocfd_b200 import cases, solver, surrogate
    nz = a.nz or 256
    case = cases.jet(nx=384, ny=256, nz=nz)
    name = "jet-%dx%dx%d-H2air-9sp-19reac-WENO5-CD6-Wilke" % case.shape
    sg = surrogate.Surrogate()
    t0 = time.perf_counter()
    # the jet's chemical change per step is orders of magnitude below the batch reactors', so the
    # network is trained on jet states alone (two snapshots of the run) to resolve it
    parts = [sg.flow_samples(case, 8, 1 << 20, seed=1), sg.flow_samples(case, 16, 1 << 20, seed=2)]
    hist = sg.train_on(parts, epochs=a.sg_epochs)
    train_s = time.perf_counter() - t0
    L = solver.lib()
    chk = solver._chk
    res = {}
    for mode in (0, 1):
        g = solver.Solver(case)
        g.init_state()
        if mode == 1:
            chk(L.ocfd_gpu_chem_mode(1, a.sg_tol))
        dt, tt = case.dt, 0.0
        chk(L.ocfd_gpu_run(dt, tt, a.warmup, 1, case.nsub))
        tt += a.warmup * dt
        with Clocks(0) as clk:
            chk(L.ocfd_gpu_event_record(0))
            chk(L.ocfd_gpu_run(dt, tt, a.steps, 1, case.nsub))
            chk(L.ocfd_gpu_event_record(1))
            ms = C.c_double()
            chk(L.ocfd_gpu_event_elapsed(0, 1, C.byref(ms)))
        reasons = (C.c_longlong * 5)()
        rejected = L.ocfd_gpu_chem_surrogate_rejected(reasons) if mode == 1 else 0
        f, di, prims = g.download_state()
        g.close()
        Li = 4
        T = prims[4][Li:-Li, Li:-Li, Li:-Li]
        dd = di[:, Li:-Li, Li:-Li, Li:-Li]
        Y = dd / dd.sum(axis=0, keepdims=True)
        res[mode] = dict(ms=ms.value / a.steps, T=T, Y=Y, rejected=rejected, reasons=list(reasons), clocks=clk.summary())
    T0, T1 = res[0]["T"], res[1]["T"]
    ncell = case.ncell
    out = {"metric": METRIC, "value": ncell / (res[1]["ms"] * 1e-3) / 1e6, "unit": UNIT, "n_gpus": 1,
           "steps": a.steps, "warmup": a.warmup, "ms_per_step": res[1]["ms"], "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64 flow + bf16 gated surrogate chemistry",
           "data": "synthetic (seeded)",
           "config": {"workload": name + "-surrogateChem", "cells_per_gpu": ncell, "dt": case.dt,
                      "train": "2 x 2^20 cells of jet snapshots after 8 and 16 steps, %d epochs, %.0f s" %
                               (a.sg_epochs, train_s),
                      "loss_first_last": [float(hist[0]), float(hist[-1])], "tol_T_K": a.sg_tol},
           "plain_fp64": {"value": ncell / (res[0]["ms"] * 1e-3) / 1e6, "ms_per_step": res[0]["ms"]},
           "speedup_vs_plain": res[0]["ms"] / res[1]["ms"],
           "accuracy_vs_plain_after_steps": {
               "steps": a.warmup + a.steps,
               "peak_T_rel_err": float(abs(T1.max() - T0.max()) / T0.max()),
               "T_err_max_K": float(np.abs(T1 - T0).max()),
               "Y_err_max": float(np.abs(res[1]["Y"] - res[0]["Y"]).max())},
           "rejected_cells_last_call": int(res[1]["rejected"]),
           "rejection_reasons": dict(zip(["negative_Y", "T_check", "T_range", "logp_range", "logdt_range"],
                                         res[1]["reasons"])),
           "clocks": res[1]["clocks"], "cpu_baseline": None, "e2e": None, "gpu_launches": None}
    print(json.dumps(out))
    return 0


def main_ours(a):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        devs = vis.split(",") if vis else [str(i) for i in range(64)]
        os.environ["CUDA_VISIBLE_DEVICES"] = devs[local]
    import numpy as np
    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(0)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from ocfd_b200 import abi, solver
    L = solver.lib()
    import ctypes as C

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    c, name = make_case(a.workload, nz=a.nz)
    if a.character:
        c.params.if_scheme_character = 1
        name += "-characteristic"
    g = solver.Solver(c)
    state_gb = L.ocfd_gpu_device_bytes() / 1e9
    g.init_state()
    dt = c.dt
    tt = 0.0
    chk = solver._chk
    reac, nsub = int(getattr(c, "if_reaction", 0) or 0), int(getattr(c, "nsub", 1) or 1)
    tiles = {"mode": a.tiles, "choice": g.tiles()}
    if a.tiles not in ("auto", "default"):
        g.set_tiles([int(x) for x in a.tiles.split(",")])
        tiles = {"mode": "given", "choice": g.tiles()}
    elif a.tiles == "auto":
        chk(L.ocfd_gpu_run(dt, tt, 1, reac, nsub))  # one step so that the tuner sees a running state
        tt += dt
        choice, tms = g.autotune(reps=5)
        tiles = {"mode": "auto", "choice": choice,
                 "candidate_ms": {"flux_x": tms[0:3], "flux_y": tms[3:6], "flux_z": tms[6:9],
                                  "visc_ev_kc8_16_32_64": tms[9:13],
                                  "visc_div_kc8_16_32_64_percell": tms[13:18],
                                  "stored_metrics_flux_xyz_ev_div": tms[18:23],
                                  "flow_rhs_visc_after_beside": tms[23:25]},
                 "choice_keys": ["flux_x_shape", "flux_y_shape", "flux_z_shape", "visc_ev_kc", "visc_div_kc",
                                 "flux_stored_metrics", "visc_ev_stored_metrics", "visc_div_stored_metrics",
                                 "visc_ev_second_stream"]}
    chk(L.ocfd_gpu_run(dt, tt, a.warmup, reac, nsub))
    tt += a.warmup * dt

    # ---- device-resident throughput ----
    barrier()
    l0 = L.ocfd_gpu_launch_count()
    with Clocks(0) as clk:
        profiler(True, a.profile_region)
        chk(L.ocfd_gpu_event_record(0))
        chk(L.ocfd_gpu_run(dt, tt, a.steps, reac, nsub))
        chk(L.ocfd_gpu_event_record(1))
        profiler(False, a.profile_region)
        ms = C.c_double()
        chk(L.ocfd_gpu_event_elapsed(0, 1, C.byref(ms)))
    tt += a.steps * dt
    launches = L.ocfd_gpu_launch_count() - l0
    barrier()
    el_ms = max_over_ranks(ms.value)
    value = world * c.ncell * a.steps / (el_ms * 1e-3) / 1e6

    # ---- roofline: per-kernel-class event timing of 2 plain-launch steps ----
    solver.Solver.profile(True)
    for s in range(2):
        g.tt = tt
        g.step(dt, reac, nsub)
        tt += dt
    prof = solver.Solver.profile_read()
    solver.Solver.profile(False)
    step_ms = sum(v[0] for v in prof.values()) / 2.0
    dom = max((k for k in prof if k in ALG_BYTES_PER_CELL), key=lambda k: prof[k][0])
    dom_ms = prof[dom][0] / max(prof[dom][1], 1)
    hbm, hbm_kind = peaks()
    alg = ALG_BYTES_PER_CELL[dom] * c.ncell
    achieved = alg / (dom_ms * 1e-3) / 1e9
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic_per_cell.json")
    if os.path.exists(tfile):
        with open(tfile) as fh:
            tr = json.load(fh)
        if dom in tr:
            traffic = tr[dom] * c.ncell
    fp64 = solver.fp64_peak_gflops()
    # the build keeps multiplies and adds separate (no FMA), so the FP64 operation peak is half
    # the measured FMA flop rate
    fp64_ops_peak = fp64 / 2.0
    fp64_roof = None
    if a.workload == "flatplate" and dom in ALG_FLOPS_PER_CELL:
        ops = ALG_FLOPS_PER_CELL[dom] * c.ncell
        ach = ops / (dom_ms * 1e-3) / 1e9
        fp64_roof = {"achieved": ach, "peak": fp64_ops_peak, "unit": "GFLOP/s", "frac": ach / fp64_ops_peak,
                     "alg_flops_per_launch": ops, "peak_kind": "measured FP64 FMA rate / 2 (no-FMA build)"}
    roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "traffic": traffic, "peak_kind": hbm_kind,
            "alg_bytes_per_launch": alg, "avg_launch_ms": dom_ms,
            "share_of_step": prof[dom][0] / 2.0 / step_ms if step_ms > 0 else None,
            "fp64": fp64_roof,
            "fp64_fma_peak_gflops_measured": fp64,
            "kernel_shares": {k: round(v[0] / 2.0 / step_ms, 4) for k, v in prof.items() if v[1] > 0}}

    # ---- e2e through the C ABI with host buffers ----
    e2e = None
    if not a.no_e2e:
        nx, ny, nz = c.shape
        hs = c.halo_shape()
        H = hs[0] * hs[1] * hs[2]
        N = c.ncell
        ns = c.params.n_spec
        nbytes_f, nbytes_di, nbytes_pr = 8 * 5 * N, 8 * ns * H, 8 * 7 * H
        bufs = []

        def pinned(nb, shape):
            p = C.c_void_p()
            chk(L.ocfd_gpu_pinned_alloc(nb, C.byref(p)))
            bufs.append(p)
            arr = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double)), shape=shape)
            return arr

        hf = pinned(nbytes_f, (5, nz, ny, nx))
        hdi = pinned(nbytes_di, (ns,) + hs)
        hpr = pinned(nbytes_pr, (7,) + hs)
        chk(L.ocfd_gpu_download_state(abi.dptr(hf), abi.dptr(hdi), abi.dptr(hpr)))
        barrier()
        chk(L.ocfd_gpu_event_record(2))
        for s in range(a.e2e_steps):
            chk(L.ocfd_gpu_upload_state(abi.dptr(hf), abi.dptr(hdi), abi.dptr(hpr)))
            chk(L.ocfd_gpu_run(dt, tt, 1, reac, nsub))
            tt += dt
            chk(L.ocfd_gpu_download_state(abi.dptr(hf), abi.dptr(hdi), None))
        chk(L.ocfd_gpu_event_record(3))
        ms2 = C.c_double()
        chk(L.ocfd_gpu_event_elapsed(2, 3, C.byref(ms2)))
        e2e_ms = max_over_ranks(ms2.value)
        e2e = {"value": world * N * a.e2e_steps / (e2e_ms * 1e-3) / 1e6, "unit": UNIT,
               "h2d_bytes_per_step": nbytes_f + nbytes_di + nbytes_pr, "d2h_bytes_per_step": nbytes_f + nbytes_di,
               "steps": a.e2e_steps}
        for p in bufs:
            L.ocfd_gpu_pinned_free(p)
    g.close()

    # ---- CPU baseline (rank 0, N = 1): the oracle on a bounded sample ----
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle
        cores = pyoracle.lib().ocfd_cpu_set_threads(os.cpu_count() or 1)
        if a.workload == "flatplate":
            cs, _ = make_case("flatplate", nz=16)
            sample = "one time step of a 1024x160x16 slab of the workload (z periodic), after one warm-up step"
        elif a.workload == "jet":
            from ocfd_b200 import cases
            cs = cases.jet(nx=96, ny=64, nz=64)
            sample = "one reacting time step of the jet on a 96x64x64 grid (same physics), after one warm-up step"
        else:
            cs, _ = make_case("isotropic")
            sample = "one time step of the 64^3 workload after one warm-up step"
        o = pyoracle.OracleSolver(cs)
        o.init_state()
        creac, cnsub = int(getattr(cs, "if_reaction", 0) or 0), int(getattr(cs, "nsub", 1) or 1)
        o.step(cs.dt, 0.0, creac, cnsub)
        t0 = time.perf_counter()
        o.step(cs.dt, cs.dt, creac, cnsub)
        el = time.perf_counter() - t0
        o.close()
        cpu = {"value": cs.ncell / el / 1e6, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}

    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
               "warmup": a.warmup, "ms_per_step": el_ms / a.steps, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
               "config": {"workload": name, "cells_per_gpu": c.ncell, "dt": dt, "chemistry": ("plain FP64 implicit Euler, %d sub-step(s) per step" % nsub) if reac else "off (non-reacting air)",
                          "parallelism": "replicas x%d (no data-path collective)" % world,
                          "tiles": tiles,
                          "l2": "device state %.1f GB per GPU >> 126 MB L2; no flush between steps" % state_gb},
               "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
               "clocks": clk.summary()}
        print(json.dumps(out))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    a = parse()
    if a.impl == "reference":
        sys.exit(main_reference(a))
    if a.workload == "reactors":
        sys.exit(main_reactors(a) if int(os.environ.get("RANK", "0")) == 0 else 0)
    if a.workload == "surrogate":
        sys.exit(main_surrogate(a) if int(os.environ.get("RANK", "0")) == 0 else 0)
    if a.workload == "jet" and a.surrogate:
        sys.exit(main_jet_surrogate(a) if int(os.environ.get("RANK", "0")) == 0 else 0)
    sys.exit(main_ours(a))
