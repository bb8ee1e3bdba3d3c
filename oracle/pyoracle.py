"""TEST INFRASTRUCTURE ONLY -- Python binding of the CPU oracle (oracle/_build/libocfd_oracle.so).

Loaded by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm, and only
as the checker or the timed CPU baseline; the product path never imports it.
The oracle exports the same entry points as the GPU library with the prefix ocfd_cpu_.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libocfd_oracle.so")
sys.path.insert(0, os.path.join(HERE, "..", "opencfd-comb_b200"))
from ocfd_b200 import abi  # noqa: E402


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = C.CDLL(LIB)
        PD, PI = C.POINTER(C.c_double), C.POINTER(C.c_int)
        sig = {
            "ocfd_cpu_init": (C.c_int, [C.POINTER(abi.Params), C.POINTER(abi.Thermo), C.POINTER(abi.Kinetics),
                                        C.POINTER(abi.Transport), C.POINTER(abi.BcData), PD, PD]),
            "ocfd_cpu_init_state": (C.c_int, [PD, PD, C.c_double]),
            "ocfd_cpu_upload_state": (C.c_int, [PD, PD, PD]),
            "ocfd_cpu_flow_advance": (C.c_int, [C.c_double, C.c_double]),
            "ocfd_cpu_chem_advance": (C.c_int, [C.c_double, C.c_int]),
            "ocfd_cpu_step": (C.c_int, [C.c_double, C.c_double, C.c_int, C.c_int]),
            "ocfd_cpu_download_state": (C.c_int, [PD, PD, PD]),
            "ocfd_cpu_download_rhybrid": (C.c_int, [PD]),
            "ocfd_cpu_download_metrics": (C.c_int, [PD]),
            "ocfd_cpu_diag": (C.c_int, [PD, PD]),
            "ocfd_cpu_chem_batch": (C.c_int, [C.POINTER(abi.Thermo), C.POINTER(abi.Kinetics), C.c_int, C.c_int,
                                              C.c_int, PD, PD, PD, PI, C.c_int, C.c_int]),
            "ocfd_cpu_probe": (C.c_double, [C.POINTER(abi.Thermo), C.c_int, C.c_int, PD, C.c_double]),
            "ocfd_cpu_set_threads": (C.c_int, [C.c_int]),
            "ocfd_cpu_flux_line": (C.c_int, [C.c_int, C.c_int, PD, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, PI,
                                             C.c_double, C.c_double, C.c_double, PD]),
            "ocfd_cpu_split": (C.c_int, [C.c_int, PD, PD, PD]),
            "ocfd_cpu_gauss": (C.c_int, [C.c_int, PD, PD, PD]),
            "ocfd_cpu_filtering": (C.c_int, [C.c_int, C.c_int, PD, PI]),
            "ocfd_cpu_ana_box": (C.c_int, [C.c_double, PD]),
            "ocfd_cpu_ana_q": (C.c_int, [PD]),
            "ocfd_cpu_ana_time_average": (C.c_int, [C.c_double, PI, PD]),
            "ocfd_cpu_ana_average_download": (C.c_int, [PD]),
            "ocfd_cpu_neg_et": (C.c_longlong, []),
            "ocfd_cpu_last_error": (C.c_char_p, []),
            "ocfd_cpu_finalize": (C.c_int, []),
        }
        for name, (res, args) in sig.items():
            fn = getattr(_lib, name)
            fn.restype = res
            fn.argtypes = args
    return _lib


class OracleError(RuntimeError):
    pass


def _chk(rc):
    if rc != 0:
        raise OracleError("oracle error %d: %s" % (rc, lib().ocfd_cpu_last_error().decode()))


class OracleSolver:
    """CPU oracle driven through the same call sequence as ocfd_b200.Solver."""

    def __init__(self, case, threads=0):
        L = lib()
        if threads:
            L.ocfd_cpu_set_threads(threads)
        self.case = case
        bc = case.bcdata()
        _chk(L.ocfd_cpu_init(C.byref(case.params), C.byref(case.thermo),
                             C.byref(case.kin) if case.kin is not None else None, C.byref(case.trans),
                             C.byref(bc) if bc is not None else None, abi.dptr(case.coords), None))
        hz, hy, hx = case.halo_shape()
        self.H = hz * hy * hx

    def init_state(self, tt=0.0):
        c = self.case
        _chk(lib().ocfd_cpu_init_state(abi.dptr(c.prim5), abi.dptr(c.di), tt))

    def upload_state(self, f, di, prims):
        _chk(lib().ocfd_cpu_upload_state(abi.dptr(f), abi.dptr(di), abi.dptr(prims)))

    def flow_time_advance(self, dt1, tt=0.0):
        _chk(lib().ocfd_cpu_flow_advance(dt1, tt))

    def chemical_time_advance(self, dt2, nsub=1):
        _chk(lib().ocfd_cpu_chem_advance(dt2, nsub))

    def step(self, dt, tt=0.0, if_reaction=0, nsub=1):
        _chk(lib().ocfd_cpu_step(dt, tt, if_reaction, nsub))

    def download_state(self):
        c = self.case
        nx, ny, nz = c.shape
        hs = c.halo_shape()
        ns = c.params.n_spec
        f = np.empty((5, nz, ny, nx))
        di = np.empty((ns,) + hs)
        prims = np.empty((7,) + hs)
        _chk(lib().ocfd_cpu_download_state(abi.dptr(f), abi.dptr(di), abi.dptr(prims)))
        return f, di, prims

    def rhybrid(self):
        r = np.empty(self.case.halo_shape())
        _chk(lib().ocfd_cpu_download_rhybrid(abi.dptr(r)))
        return r

    def metrics(self):
        m = np.empty((10,) + self.case.halo_shape())
        _chk(lib().ocfd_cpu_download_metrics(abi.dptr(m)))
        return m

    def diag(self):
        e, k = C.c_double(), C.c_double()
        _chk(lib().ocfd_cpu_diag(C.byref(e), C.byref(k)))
        return e.value, k.value

    # ---- filtering and analysis (code/others/OCFD_filtering.f90, OCFD_ANA.f90) ----
    def filtering(self, istep, table, nfiltering):
        """table: Para%Filter as a (10, 100) array (row m = filter group m), see post.filter_table."""
        t = np.ascontiguousarray(table, dtype=np.float64)
        applied = C.c_int()
        _chk(lib().ocfd_cpu_filtering(istep, nfiltering, abi.dptr(t), C.byref(applied)))
        return applied.value

    def ana_box(self, tt):
        out = np.empty(19)
        _chk(lib().ocfd_cpu_ana_box(tt, abi.dptr(out)))
        return out

    def ana_q(self):
        nx, ny, nz = self.case.shape
        q = np.empty((nz, ny, nx))
        _chk(lib().ocfd_cpu_ana_q(abi.dptr(q)))
        return q

    def ana_time_average(self, dt):
        k, t = C.c_int(), C.c_double()
        _chk(lib().ocfd_cpu_ana_time_average(dt, C.byref(k), C.byref(t)))
        return k.value, t.value

    def ana_average(self):
        nx, ny, nz = self.case.shape
        a = np.empty((5 + self.case.params.n_spec, nz, ny, nx))
        _chk(lib().ocfd_cpu_ana_average_download(abi.dptr(a)))
        return a

    def close(self):
        lib().ocfd_cpu_finalize()


def chem_batch(thermo, kin, realgas, timeadv, di, e, dt, nsub=None, threads=0, const_p=False):
    """Batched 0-D reactors on the CPU; di (n, Ns) and e (n) are updated in place. const_p: hold
    each reactor's initial pressure at constant specific enthalpy after every sub-step (an
    extension; the reference's reactor is constant-volume)."""
    n = len(e)
    _chk(lib().ocfd_cpu_chem_batch(C.byref(thermo), C.byref(kin), realgas, timeadv, n, abi.dptr(di), abi.dptr(e),
                                   abi.dptr(dt), abi.iptr(nsub), threads, 1 if const_p else 0))


def flux_line(scheme, plus, f, bnd=(0, 0), sb=(0, 0), scm=None, ud7l_diss=1.0, theta=(1.0, 1.0)):
    """Numerical fluxes hh(0:n) of one pencil f(1-LAP:n+LAP) (length n+8)."""
    f = np.ascontiguousarray(f, dtype=np.float64)
    n = len(f) - 8
    hh = np.zeros(n + 1)
    sc = None if scm is None else np.ascontiguousarray(scm, dtype=np.int32)
    lib().ocfd_cpu_flux_line(scheme, 1 if plus else 0, abi.dptr(f), n, bnd[0], bnd[1], sb[0], sb[1],
                             abi.iptr(sc), ud7l_diss, theta[0], theta[1], abi.dptr(hh))
    return hh


def split(kind, Et, p, d, u, v, w, A1, A2, A3):
    inp = np.array([Et, p, d, u, v, w, A1, A2, A3], dtype=np.float64)
    fp = np.zeros(5)
    fm = np.zeros(5)
    lib().ocfd_cpu_split(kind, abi.dptr(inp), abi.dptr(fp), abi.dptr(fm))
    return fp, fm


def gauss(A, b):
    A = np.ascontiguousarray(A, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros(len(b))
    lib().ocfd_cpu_gauss(len(b), abi.dptr(A), abi.dptr(b), abi.dptr(x))
    return x


def probe(thermo, realgas, what, di, x):
    di = np.ascontiguousarray(di, dtype=np.float64)
    return lib().ocfd_cpu_probe(C.byref(thermo), realgas, what, abi.dptr(di), x)
