"""Throughput of the OpenCFD-Comb hot path on B200: Mcell-steps/s of whole reference time steps
(two RK3 flow half-steps with the finite-rate chemistry between them).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload jet|flatplate|isotropic|reactors|surrogate]
  python bench.py --impl reference ...      (the reference algorithm on the host cores)

Workload (default): the 3-D reacting H2 jet into hot air coflow, 384x256x256 cells, 9 species and
19 reactions, WENO5 Steger-Warming inviscid flux, CD6 viscous terms, Wilke transport, FP64
implicit-Euler chemistry, BC_JET inflow with seeded 2 % velocity noise. The same process runs
the jet twice from the same start: once with the plain FP64 chemistry integrator and once with
the gated BF16 chemistry surrogate (trained first, on the GPU, on cells of an FP64 run). `value` is
the plain FP64 form; the `surrogate` object holds the surrogate form's throughput, its speed-up
over the plain form, its fallback fraction and its temperature and species errors against the
plain FP64 run after the configured 200 steps. The flat plate (1024x160x128, HYBRID) is
`--workload flatplate`.

Multi-GPU runs are independent replicas (one per rank, weak scaling): the single-rank solver has
no exchange step, so no collective is invented; ranks meet only for the timing barrier and the
max-over-ranks reduction.

The device-resident number (value) times K graph-replayed steps with CUDA events on the library
stream; the state (tens of GB) is far larger than the 126 MB L2, so no flush is needed. e2e times
steps through the C ABI with the state uploaded from pinned host memory and the conserved
variables and species densities downloaded every step. The roofline object names the kernel
class with the largest share of a step, timed live with per-launch CUDA events.
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
    ap.add_argument("--lib", default="fma", choices=["fma", "exact"],
                    help="library build: fma = contracted multiply-adds (libocfd_gpu_fma.so, checked against the "
                         "CPU restatement to 1e-10 after ten steps with identical HYBRID decisions), exact = "
                         "--fmad=false (libocfd_gpu.so, bit-identical to it where no transcendental enters)")
    ap.add_argument("--workload", default="jet", choices=["jet", "flatplate", "isotropic", "reactors", "surrogate"],
                    help="jet = the metric's configuration (384x256x256 reacting H2 jet, plain FP64 and gated "
                         "surrogate chemistry); flatplate, isotropic, reactors and surrogate are the other "
                         "configurations (1024x160x128 M2.25 flat plate, 64^3 decaying turbulence, 2^20 batched "
                         "0-D reactors, the surrogate on 2^20 held-out reactors)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--sg-train", type=int, default=1 << 22,
                    help="surrogate workload: C3 reactors drawn (two trajectory states each)")
    ap.add_argument("--sg-jet-cells", type=int, default=1 << 21, help="surrogate workload: jet snapshot cells")
    ap.add_argument("--sg-epochs", type=int, default=None,
                    help="training epochs (default: 20 for the jet's training set, 6 for the surrogate workload)")
    ap.add_argument("--sg-batch", type=int, default=4096, help="surrogate workload: training batch")
    ap.add_argument("--sg-tol", type=float, default=5.0, help="surrogate workload: gate tolerance on T (K)")
    ap.add_argument("--const-v", action="store_true",
                    help="reactors workload: the reference's constant-volume reactor instead of the configured "
                         "constant-pressure one")
    ap.add_argument("--no-surrogate", action="store_true",
                    help="jet workload: plain FP64 chemistry only (no surrogate training or second run)")
    ap.add_argument("--total-steps", type=int, default=200,
                    help="jet workload: steps of each run (plain and surrogate) after which the errors are taken")
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
    Fortran compiler exists on this image, so the reference binary itself cannot be built). Each
    timed step is one full time step of a bounded sample of the workload, on all host threads."""
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    cores = pyoracle.lib().ocfd_cpu_set_threads(os.cpu_count() or 1)
    if a.workload in ("reactors", "surrogate"):  # the reference has only the FP64 integrator
        return reactors_reference(a, pyoracle, cores)
    if a.workload == "flatplate":
        # size the slab so that warmup + steps take about two minutes
        probe, _ = make_case(a.workload, nz=8)
        o = pyoracle.OracleSolver(probe)
        o.init_state()
        t0 = time.perf_counter()
        o.step(probe.dt, 0.0)
        rate = probe.ncell / (time.perf_counter() - t0)
        o.close()
        nz = int(max(8, min(128, 120.0 * rate / (1024 * 160 * (a.steps + a.warmup)))))
        c, name = make_case(a.workload, nz=nz)
        full_name = make_case(a.workload)[1]
        sample = "per step: one full time step of a 1024x160x%d slab of the 1024x160x128 workload (z periodic)" % nz
    elif a.workload == "jet":
        from ocfd_b200 import cases
        c = cases.jet(nx=96, ny=64, nz=64)
        name = "jet-96x64x64-H2air-9sp-19reac-WENO5-CD6-SW-Wilke-implicitChem"
        full_name = "jet-384x256x256-H2air-9sp-19reac-WENO5-CD6-SW-Wilke-implicitChem"
        sample = ("per step: one reacting time step (plain FP64 chemistry) of the jet on a 96x64x64 grid (same "
                  "physics and inflow as the 384x256x256 workload)")
    else:
        c, name = make_case(a.workload)
        full_name = name
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
           "config": {"workload": name, "sample_of": full_name, "sample_cells": c.ncell,
                      "chemistry": "plain FP64 implicit Euler" if reac else "off"},
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
    cp = a.workload == "reactors" and not a.const_v
    names, th, kin, di, E, dt, nsub, T = cases.reactors(n=n, seed=1)
    for s in range(a.warmup):
        pyoracle.chem_batch(th, kin, 1, abi.CHEM_IMPLICIT, di.copy(), E.copy(), dt, nsub, const_p=cp)
    t0 = time.perf_counter()
    for s in range(a.steps):
        pyoracle.chem_batch(th, kin, 1, abi.CHEM_IMPLICIT, di.copy(), E.copy(), dt, nsub, const_p=cp)
    el = time.perf_counter() - t0
    val = n * a.steps / el / 1e6
    out = {"metric": RMETRIC, "value": val, "unit": RUNIT, "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
           "ms_per_step": el * 1e3 / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64", "data": "synthetic (seeded)", "impl": "reference",
           "config": {"workload": "reactors-%d-H2air-9sp-implicitEuler-%s" % (n, "constP" if cp else "constV"),
                      "sample_of": "reactors-2^20-H2air-9sp-implicitEuler", "sample_reactors": n},
           "cpu_baseline": {"value": val, "unit": RUNIT, "cores": cores, "kind": "port",
                            "sample": "per step: %d reactors drawn like the 2^20 workload" % n},
           "e2e": {"value": val, "unit": RUNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


def main_reactors(a):
    """2^20 independent H2-air reactors at 1 atm (constant-pressure as configured, or the
    reference's constant-volume reactor with --const-v) through the persistent work-queue kernel
    (ocfd_gpu_chem_batch_device); one step = one pass over all reactors."""
    import numpy as np
    import torch
    from ocfd_b200 import abi, cases, solver
    L = solver.lib()
    import ctypes as C
    n = 2 ** 20
    names, th, kin, di, E, dt, nsub, T = cases.reactors(n=n, seed=0)
    cp = not a.const_v
    solver.chem_setup(th, kin, 1, abi.CHEM_IMPLICIT, const_p=cp)
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
        pyoracle.chem_batch(th, kin, 1, abi.CHEM_IMPLICIT, sdi.copy(), sE.copy(), sdt, sns, const_p=cp)
        el = time.perf_counter() - t0
        cpu = {"value": m / el / 1e6, "unit": RUNIT, "cores": cores, "kind": "port",
               "sample": "%d reactors drawn like the 2^20 workload" % m}
    sub = int(nsub.sum())
    out = {"metric": RMETRIC, "value": value, "unit": RUNIT, "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
           "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64", "data": "synthetic (seeded)",
           "config": {"workload": "reactors-2^20-H2air-9sp-implicitEuler-%s" % ("constP" if cp else "constV"),
                      "reactor": "constant-pressure (p held at constant specific enthalpy after every sub-step)"
                                 if cp else "constant-volume (the reference's)", "reactors": n, "substeps_total": sub,
                      "substeps_per_s": sub * a.steps / (ms * 1e-3),
                      "l2": "inputs re-copied from a pristine device copy before each pass"},
           "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": None, "clocks": clk.summary()}
    print(json.dumps(out))
    return 0


# ---------------------------------------------------------------- surrogate chemistry (C4)
SMETRIC = "Mreactor-solves/s on 1 B200: plain FP64 vs gated surrogate chemistry at <=1% T error, 2^20 H2-air reactors"
MLP_FLOPS_PER_SAMPLE = 2 * (16 * 256 + 256 * 256 * 2 + 256 * 16)  # padded forward pass


def main_surrogate(a):
    """C4: the learned chemistry on its configured state set. 10 x 2^20 states (C3 reactors at two
    points of their FP64 constant-pressure trajectory, 2^23 states, plus 2^21 cells of two FP64 jet
    snapshots) are split 90/10 with a seeded permutation; the network is trained on the 90 % with
    FP64-integrator targets, then the plain FP64 batch and the gated surrogate are timed on the 2^20
    held-out states (device-resident inputs restored before every pass) and the surrogate's errors
    against the FP64 integrator and its fallback fraction are taken on them."""
    import numpy as np
    import torch
    import ctypes as C
    from ocfd_b200 import solver, surrogate
    sg = surrogate.Surrogate()
    L = sg.L
    t0 = time.perf_counter()
    ADI, AE, ADT, ANS, SRC = sg.c4_states(n_reactors=a.sg_train, jet_cells=a.sg_jet_cells, seed=0)
    ntot = len(AE)
    n = 1 << 20
    tr, ho = sg.split(ntot, n, seed=0)
    build_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    hist = sg.train_on([(ADI[tr], AE[tr], ADT[tr], ANS[tr])], epochs=a.sg_epochs, batch=a.sg_batch, lr=2e-3, seed=0)
    train_s = time.perf_counter() - t0
    di, E, dt, nsub = (np.ascontiguousarray(x[ho]) for x in (ADI, AE, ADT, ANS))
    held_jet = int(SRC[ho].sum())
    del ADI, AE, ADT, ANS
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
    acc = sg.evaluate_on(di, E, dt, nsub, tol_T=a.sg_tol)
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
           "config": {"workload": "surrogate-2^20-held-out-states-H2air-9sp (MLP 12-256-256-256-10, GELU)",
                      "states": ntot, "train_states": len(tr), "held_out_states": n,
                      "held_out_from_jet": held_jet, "held_out_from_reactors": n - held_jet,
                      "state_set": "2 x %d C3 reactor states (draw, and after one FP64 constant-pressure "
                                   "integration over dt) + %d cells of two FP64 jet snapshots (384x256x256, "
                                   "steps 8 and 16); seeded 90/10 split" % (a.sg_train, a.sg_jet_cells),
                      "targets": "FP64 implicit-Euler integrator (constant volume, the operator the surrogate "
                                 "replaces) over each state's dt",
                      "epochs": a.sg_epochs, "batch": a.sg_batch, "build_seconds": build_s,
                      "train_seconds": train_s,
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


# algorithmic bytes per cell and RK stage of each kernel class on the reacting jet (N_SPEC = 9,
# FP64; every input read once, every output written once; the grid is a tensor product, so the
# metrics are 1-D arrays and count as 0). A class of several launches per stage counts them all:
#  flux_x / flux_y / flux_z : read d,u,v,w,p,Et (6); write du (5), y / z also read du (5)
#  visc_ev : read u,v,w,T,Amu,Amk,Qp(3) (9); write Ev1..Ev3 (12)                      = 21 doubles
#  visc_div: read Ev (12); read + write du(2..5) (8)                                   = 20
#  rk_prims: read f,fn,du (15), di (9); write f (5), d,u,v,w,T,p,Et (7), di (9)        = 45
#  transport (k_transport): read d,T,p,di(9) (12); write Amu, Amk, AmD(9) (11)         = 23
#  species_flux (x, y, z scalar sweeps): read di(9),u,v,w; write Dus(9); y, z read Dus = 81
#  species_visc: k_ci read di(9),d, write ci(9) (19); k_scal_ev read ci(9),d,T,AmD(9),
#    write Ev(27),Qp(3) (50); k_scal_div read Ev(27), read + write Dus(9) (45)         = 114
#  species_rk (k_scal_rk): read Dus(9), din(9), di(9); write di(9)                      = 36
#  chem (once per step, k_chem_cells): read + write di(9), Et, f5; read T, p            = 22
# species_visc: k_ci + k_scal_ev + k_scal_div with the species RK update fused in (912 B of the
# viscous kernels + 288 B of the update - the 144 B of Dus that no longer travel)
JET_ALG_BYTES = {"flux_x": 88, "flux_y": 128, "flux_z": 128, "visc_ev": 168, "visc_div": 160, "rk_prims": 360,
                 "transport": 184, "species_flux": 648, "species_visc": 1056, "species_rk": 288}
JET_CHEM_BYTES = 176
JET_STAGES_PER_STEP = 6


class Ranks:
    """One process per GPU under torchrun (replicas): NCCL only for the timing barrier and the
    max-over-ranks reduction."""

    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        local = int(os.environ.get("LOCAL_RANK", "0"))
        if self.world > 1:
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            devs = vis.split(",") if vis else [str(i) for i in range(64)]
            os.environ["CUDA_VISIBLE_DEVICES"] = devs[local]
        import torch
        self.torch = torch
        self.dist = None
        if self.world > 1:
            import datetime
            import torch.distributed as dist
            torch.cuda.set_device(0)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
            self.dist = dist

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()
        self.torch.cuda.synchronize()

    def max(self, x):
        if self.dist is None:
            return x
        t = self.torch.tensor([x], dtype=self.torch.float64, device="cuda")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()


def merge_clocks(*cs):
    sm = [x for c in cs for x in ([c["sm_mhz"]] if c.get("sm_mhz") else [])]
    mx = [c["sm_max_mhz"] for c in cs if c.get("sm_max_mhz")]
    return {"sm_mhz": min(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
            "reasons": sorted({r for c in cs for r in c.get("reasons", [])}),
            "samples": sum(c.get("samples", 0) for c in cs)}


def timed_run(L, dt, tt, k, reac, nsub):
    """K graph-replayed steps between two CUDA events on the library stream; (ms, launches, clocks)."""
    import ctypes as C
    from ocfd_b200 import solver
    chk = solver._chk
    l0 = L.ocfd_gpu_launch_count()
    with Clocks(0) as clk:
        chk(L.ocfd_gpu_event_record(0))
        chk(L.ocfd_gpu_run(dt, tt, k, reac, nsub))
        chk(L.ocfd_gpu_event_record(1))
        ms = C.c_double()
        chk(L.ocfd_gpu_event_elapsed(0, 1, C.byref(ms)))
    return ms.value, L.ocfd_gpu_launch_count() - l0, clk.summary()


def e2e_steps(L, c, dt, tt, nsteps, reac, nsub, ranks):
    """nsteps steps through the C ABI with host buffers: every step uploads the state (f, di and
    the primitives) from pinned host memory, runs the step and downloads f and di."""
    import ctypes as C
    import numpy as np
    from ocfd_b200 import abi, solver
    chk = solver._chk
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
        return np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double)), shape=shape)

    hf = pinned(nbytes_f, (5, nz, ny, nx))
    hdi = pinned(nbytes_di, (ns,) + hs)
    hpr = pinned(nbytes_pr, (7,) + hs)
    chk(L.ocfd_gpu_download_state(abi.dptr(hf), abi.dptr(hdi), abi.dptr(hpr)))
    ranks.barrier()
    chk(L.ocfd_gpu_event_record(2))
    for s in range(nsteps):
        chk(L.ocfd_gpu_upload_state(abi.dptr(hf), abi.dptr(hdi), abi.dptr(hpr)))
        chk(L.ocfd_gpu_run(dt, tt, 1, reac, nsub))
        tt += dt
        chk(L.ocfd_gpu_download_state(abi.dptr(hf), abi.dptr(hdi), None))
    chk(L.ocfd_gpu_event_record(3))
    ms = C.c_double()
    chk(L.ocfd_gpu_event_elapsed(2, 3, C.byref(ms)))
    e2e_ms = ranks.max(ms.value)
    for p in bufs:
        L.ocfd_gpu_pinned_free(p)
    return {"value": ranks.world * N * nsteps / (e2e_ms * 1e-3) / 1e6, "unit": UNIT,
            "h2d_bytes_per_step": nbytes_f + nbytes_di + nbytes_pr, "d2h_bytes_per_step": nbytes_f + nbytes_di,
            "steps": nsteps}, tt


def cpu_sample(workload):
    """The oracle (C++ restatement of the reference's Fortran) on all host threads: one time step
    of a bounded sample of the workload after one warm-up step."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    cores = pyoracle.lib().ocfd_cpu_set_threads(os.cpu_count() or 1)
    if workload == "flatplate":
        cs, _ = make_case("flatplate", nz=16)
        sample = "one time step of a 1024x160x16 slab of the workload (z periodic), after one warm-up step"
    elif workload == "jet":
        from ocfd_b200 import cases
        cs = cases.jet(nx=96, ny=64, nz=64)
        sample = ("one reacting time step (plain FP64 chemistry) of the jet on a 96x64x64 grid (same physics and "
                  "inflow), after one warm-up step")
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
    return {"value": cs.ncell / el / 1e6, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}


def jet_roofline(prof, nsteps, ncell):
    """Per-class device time of nsteps plain-launch steps (per-launch CUDA events) against the
    classes' algorithmic bytes; the roofline object is the class with the largest share."""
    hbm, hbm_kind = peaks()
    step_ms = sum(v[0] for v in prof.values()) / nsteps
    classes = {}
    for k, (ms, n) in prof.items():
        if n == 0:
            continue
        ms_step = ms / nsteps
        row = {"ms_per_step": round(ms_step, 4), "launches_per_step": n / nsteps,
               "share_of_step": round(ms_step / step_ms, 4) if step_ms > 0 else None}
        alg = None
        if k in JET_ALG_BYTES:
            alg = JET_ALG_BYTES[k] * JET_STAGES_PER_STEP * ncell
        elif k == "chem":
            alg = JET_CHEM_BYTES * ncell
        if alg is not None:
            gbs = alg / (ms_step * 1e-3) / 1e9
            row.update({"alg_bytes_per_step": alg, "achieved_gbs": round(gbs, 1), "frac": round(gbs / hbm, 4)})
        classes[k] = row
    dom = max((k for k in classes if "achieved_gbs" in classes[k]), key=lambda k: classes[k]["ms_per_step"])
    d = classes[dom]
    launches = d["launches_per_step"]
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic_per_cell_jet.json")
    if os.path.exists(tfile):
        with open(tfile) as fh:
            tr = json.load(fh)
        if dom in tr:  # per launch; the file holds one stage's bytes for the classes of several launches
            per_stage = dom in ("species_flux", "species_visc")
            traffic = tr[dom] * ncell / (launches / JET_STAGES_PER_STEP if per_stage else 1.0)
    # the same class against the measured FP64 peak (FMA = 2 FLOP), with the executed FP64 operations
    # per cell that ncu counted for it (the kernels of this path are FP64-issue or latency bound)
    fp64 = None
    ffile = os.path.join(ROOT, "profiles", "fp64_flops_per_cell_jet.json")
    if os.path.exists(ffile):
        from ocfd_b200 import solver
        with open(ffile) as fh:
            fl = json.load(fh)
        if dom in fl:
            per_stage = dom in ("species_flux", "species_visc")
            flops_step = fl[dom] * ncell * (JET_STAGES_PER_STEP if per_stage else launches)
            ach = flops_step / (d["ms_per_step"] * 1e-3) / 1e9
            pk = solver.fp64_peak_gflops()
            fp64 = {"achieved": round(ach, 1), "peak": round(pk, 1), "unit": "GFLOP/s", "frac": round(ach / pk, 4),
                    "flops_per_step": flops_step, "peak_kind": "measured FP64 FMA loop (FMA = 2 FLOP)"}
    return {"bound": "hbm", "kernel": dom, "achieved": d["achieved_gbs"], "peak": hbm, "unit": "GB/s",
            "frac": d["frac"], "traffic": traffic, "peak_kind": hbm_kind, "fp64": fp64,
            "alg_bytes_per_launch": d["alg_bytes_per_step"] / launches,
            "avg_launch_ms": d["ms_per_step"] / launches, "share_of_step": d["share_of_step"],
            "note": "a class of several kernels (species_flux, species_visc) counts one stage's launches "
                    "together: achieved = their algorithmic bytes / their summed device time",
            "classes": classes}


def main_jet(a):
    """C5: the reacting jet with plain FP64 chemistry (value, e2e, roofline) and with the gated
    surrogate (trained first on cells of an FP64 run), both for the same number of steps from the
    same start, the surrogate's errors taken against the plain run at the end."""
    ranks = Ranks()
    import numpy as np
    import ctypes as C
    from ocfd_b200 import cases, solver, surrogate
    L = solver.lib()
    chk = solver._chk
    nz = a.nz or 256
    case = cases.jet(nx=384, ny=256, nz=nz)
    name = "jet-%dx%dx%d-H2air-9sp-19reac-WENO5-CD6-SW-Wilke-implicitChem" % case.shape
    dt, nsub, N = case.dt, case.nsub, case.ncell
    n_e2e = 0 if a.no_e2e else max(1, min(a.e2e_steps, 5))
    n_prof = 2
    total = max(a.total_steps, 1 + a.warmup + a.steps + n_prof + n_e2e)

    # ---- surrogate training set: cells of an FP64 run after 8 and 16 steps ----
    sg, train = None, None
    if not a.no_surrogate:
        sg = surrogate.Surrogate()
        t0 = time.perf_counter()
        g = solver.Solver(case)
        g.init_state()
        parts = []
        for s0, s1, seed in ((0, 8, 1), (8, 16, 2)):
            chk(L.ocfd_gpu_run(dt, s0 * dt, s1 - s0, 1, nsub))
            _, di, prims = g.download_state()
            parts.append(sg.samples_from_state(case, di, prims, 1 << 20, seed))
        g.close()
        hist = sg.train_on(parts, epochs=a.sg_epochs)
        train = {"cells": sum(len(p[1]) for p in parts), "epochs": a.sg_epochs,
                 "source": "2 x 2^20 cells of the plain FP64 jet run after 8 and 16 steps (seeded choice)",
                 "seconds": round(time.perf_counter() - t0, 1),
                 "loss_first_last": [float(hist[0]), float(hist[-1])]}

    # ---- plain FP64 chemistry: tune, warm up, K timed steps, roofline, e2e, up to `total` ----
    g = solver.Solver(case)
    state_gb = L.ocfd_gpu_device_bytes() / 1e9
    g.init_state()
    tt, done = 0.0, 0
    chk(L.ocfd_gpu_run(dt, tt, 1, 1, nsub))  # one step so that the tuner sees a running state
    tt += dt
    done += 1
    tiles = {"mode": a.tiles, "choice": g.tiles()}
    if a.tiles == "auto":
        choice, tms = g.autotune(reps=5)
        tiles = {"mode": "auto", "choice": choice,
                 "flow_rhs_visc_after_beside_ms": tms[23:25],
                 "stage_rhs_species_in_order_beside_ms": tms[25:27]}
    elif a.tiles != "default":
        g.set_tiles([int(x) for x in a.tiles.split(",")])
        tiles = {"mode": "given", "choice": g.tiles()}
    chk(L.ocfd_gpu_run(dt, tt, a.warmup, 1, nsub))
    tt += a.warmup * dt
    done += a.warmup
    ranks.barrier()
    ms, launches, clk_plain = timed_run(L, dt, tt, a.steps, 1, nsub)
    ranks.barrier()
    tt += a.steps * dt
    done += a.steps
    el_ms = ranks.max(ms)
    value = ranks.world * N * a.steps / (el_ms * 1e-3) / 1e6
    solver.Solver.profile(True)
    for s in range(n_prof):
        g.tt = tt
        g.step(dt, 1, nsub)
        tt += dt
    prof = solver.Solver.profile_read()
    solver.Solver.profile(False)
    done += n_prof
    roof = jet_roofline(prof, n_prof, N)
    e2e = None
    if n_e2e:
        e2e, tt = e2e_steps(L, case, dt, tt, n_e2e, 1, nsub, ranks)
        done += n_e2e
    if total > done:
        chk(L.ocfd_gpu_run(dt, tt, total - done, 1, nsub))
        tt += (total - done) * dt
    _, di0, pr0 = g.download_state()
    g.close()
    Li = 4
    T0 = pr0[4][Li:-Li, Li:-Li, Li:-Li].copy()
    d0 = di0[:, Li:-Li, Li:-Li, Li:-Li]
    Y0 = d0 / d0.sum(axis=0, keepdims=True)
    del di0, pr0, d0
    chem_share = roof["classes"].get("chem", {}).get("share_of_step")

    # ---- gated surrogate chemistry: same start, same steps ----
    sgo = None
    clk_sg = {}
    if sg is not None:
        g = solver.Solver(case)
        g.init_state()
        chk(L.ocfd_gpu_chem_mode(1, a.sg_tol))
        tt = 0.0
        chk(L.ocfd_gpu_run(dt, tt, 1, 1, nsub))
        tt += dt
        if tiles["mode"] == "auto":
            g.autotune(reps=0)  # the plain run's choice, remembered for this configuration
        else:
            g.set_tiles(tiles["choice"])
        chk(L.ocfd_gpu_run(dt, tt, a.warmup, 1, nsub))
        tt += a.warmup * dt
        ranks.barrier()
        ms_sg, _, clk_sg = timed_run(L, dt, tt, a.steps, 1, nsub)
        ranks.barrier()
        tt += a.steps * dt
        reasons = (C.c_longlong * 6)()
        rejected = L.ocfd_gpu_chem_surrogate_rejected(reasons)
        rest = total - (1 + a.warmup + a.steps)
        if rest > 0:
            chk(L.ocfd_gpu_run(dt, tt, rest, 1, nsub))
        _, di1, pr1 = g.download_state()
        g.close()
        T1 = pr1[4][Li:-Li, Li:-Li, Li:-Li]
        d1 = di1[:, Li:-Li, Li:-Li, Li:-Li]
        Y1 = d1 / d1.sum(axis=0, keepdims=True)
        ms_sg = ranks.max(ms_sg)
        peak = float(abs(T1.max() - T0.max()) / T0.max())
        yerr = float(np.abs(Y1 - Y0).max())
        sgo = {"value": ranks.world * N * a.steps / (ms_sg * 1e-3) / 1e6, "unit": UNIT,
               "ms_per_step": ms_sg / a.steps, "speedup_vs_plain": el_ms / ms_sg,
               "accuracy_vs_plain_fp64": {
                   "steps": total, "peak_T_rel_err": peak,
                   "T_err_max_K": float(np.abs(T1 - T0).max()),
                   "T_err_rel_max": float((np.abs(T1 - T0) / T0).max()),
                   "Y_err_max": yerr,
                   "target": "peak T error <= 1 %, species mass fraction error <= 1e-3",
                   "meets_target": bool(peak <= 0.01 and yerr <= 1e-3)},
               "fallback_fraction_last_step": rejected / N,
               "rejection_reasons_last_step": dict(zip(["negative_Y", "T_check", "T_range", "logp_range",
                                                         "logdt_range", "Y_range"], list(reasons))),
               "tol_T_K": a.sg_tol, "train": train,
               "chemistry_share_of_plain_step": chem_share,
               "amdahl_bound_on_speedup": (1.0 / (1.0 - chem_share)) if chem_share else None,
               "clocks": clk_sg}

    cpu = None
    if ranks.rank == 0 and ranks.world == 1 and not a.no_cpu:
        cpu = cpu_sample("jet")
    if ranks.rank == 0:
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ranks.world, "steps": a.steps,
               "warmup": a.warmup, "ms_per_step": el_ms / a.steps, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
               "value_form": "plain FP64 chemistry (implicit Euler + Gauss, the reference's integrator)",
               "config": {"workload": name, "cells_per_gpu": N, "dt": dt, "steps_per_run": total,
                          "library": os.path.basename(solver.LIBPATH),
                          "chemistry": "plain FP64 implicit Euler, %d sub-step per step; surrogate run: gated BF16 "
                                       "MLP with FP64 fallback" % nsub,
                          "parallelism": "replicas x%d (no data-path collective)" % ranks.world,
                          "tiles": tiles,
                          "l2": "device state %.1f GB per GPU >> 126 MB L2; no flush between steps" % state_gb},
               "surrogate": sgo,
               "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
               "clocks": merge_clocks(clk_plain, clk_sg) if clk_sg else clk_plain}
        print(json.dumps(out))
    ranks.close()
    return 0


def main_ours(a):
    ranks = Ranks()
    world, rank = ranks.world, ranks.rank
    import numpy as np
    from ocfd_b200 import abi, solver
    L = solver.lib()
    import ctypes as C
    barrier, max_over_ranks = ranks.barrier, ranks.max

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
                                  "flow_rhs_visc_after_beside": tms[23:25],
                                  "stage_rhs_species_in_order_beside": tms[25:27]},
                 "choice_keys": ["flux_x_shape", "flux_y_shape", "flux_z_shape", "visc_ev_kc", "visc_div_kc",
                                 "flux_stored_metrics", "visc_ev_stored_metrics", "visc_div_stored_metrics",
                                 "stream_switches (1 visc_ev beside the flux sweeps, 2 species chain on a third stream)"]}
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
    if a.workload == "jet":
        roof = jet_roofline(prof, 2, c.ncell)
    else:
        step_ms = sum(v[0] for v in prof.values()) / 2.0
        dom = max((k for k in prof if k in ALG_BYTES_PER_CELL and prof[k][1] > 0), key=lambda k: prof[k][0])
        dom_ms = prof[dom][0] / max(prof[dom][1], 1)
        hbm, hbm_kind = peaks()
        alg = ALG_BYTES_PER_CELL[dom] * c.ncell
        achieved = alg / (dom_ms * 1e-3) / 1e9
        traffic = None
        tfile = os.path.join(ROOT, "profiles", "traffic_per_cell.json")
        if os.path.exists(tfile) and a.workload == "flatplate":
            with open(tfile) as fh:
                tr = json.load(fh)
            if dom in tr:
                traffic = tr[dom] * c.ncell
        fp64 = solver.fp64_peak_gflops()
        # the exact build keeps multiplies and adds separate (no FMA), so its FP64 operation peak is
        # half the measured FMA flop rate; the contracted build is held to the full FMA flop rate
        fma_lib = solver.VARIANT == "fma"
        fp64_ops_peak = fp64 if fma_lib else fp64 / 2.0
        fp64_roof = None
        if a.workload == "flatplate" and dom in ALG_FLOPS_PER_CELL:
            ops = ALG_FLOPS_PER_CELL[dom] * c.ncell
            ach = ops / (dom_ms * 1e-3) / 1e9
            fp64_roof = {"achieved": ach, "peak": fp64_ops_peak, "unit": "GFLOP/s", "frac": ach / fp64_ops_peak,
                         "alg_flops_per_launch": ops,
                         "peak_kind": ("measured FP64 FMA loop (FMA = 2 FLOP), contracted build" if fma_lib
                                       else "measured FP64 FMA rate / 2 (no-FMA build)")}
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
        e2e, tt = e2e_steps(L, c, dt, tt, a.e2e_steps, reac, nsub, ranks)
    g.close()

    # ---- CPU baseline (rank 0, N = 1): the oracle on a bounded sample ----
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        cpu = cpu_sample(a.workload)

    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
               "warmup": a.warmup, "ms_per_step": el_ms / a.steps, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
               "config": {"workload": name, "cells_per_gpu": c.ncell, "dt": dt,
                          "library": os.path.basename(solver.LIBPATH), "chemistry": ("plain FP64 implicit Euler, %d sub-step(s) per step" % nsub) if reac else "off (non-reacting air)",
                          "parallelism": "replicas x%d (no data-path collective)" % world,
                          "tiles": tiles,
                          "l2": "device state %.1f GB per GPU >> 126 MB L2; no flush between steps" % state_gb},
               "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
               "clocks": clk.summary()}
        print(json.dumps(out))
    ranks.close()
    return 0


if __name__ == "__main__":
    a = parse()
    os.environ["OCFD_B200_LIB"] = a.lib  # read when ocfd_b200.solver is first imported
    if a.sg_epochs is None:
        a.sg_epochs = 6 if a.workload == "surrogate" else 20
    if a.impl == "reference":
        sys.exit(main_reference(a))
    if a.workload == "reactors":
        sys.exit(main_reactors(a) if int(os.environ.get("RANK", "0")) == 0 else 0)
    if a.workload == "surrogate":
        sys.exit(main_surrogate(a) if int(os.environ.get("RANK", "0")) == 0 else 0)
    if a.workload == "jet" and not a.no_surrogate:
        sys.exit(main_jet(a))
    sys.exit(main_ours(a))
