"""Host-side mirror of the reference's hot-path interface, backed by libocfd_gpu.so.

The reference's Fortran driver (code/flow-solver/OCFD_NS_Solver.f90) calls, per time step,
flow_time_advance(dt/2), Chemical_time_advance(dt/Chemical_sub_step) x Chemical_sub_step +
comput_T_P, and flow_time_advance(dt/2); show_flow_msg reduces mean energies. This class
offers the same calls (same names, argument meaning and error behaviour: a failing call raises,
as the reference stops) over the C ABI of include/ocfd_gpu.h. There is no CPU fallback: if the
CUDA library or a device is missing, construction fails.
"""
import ctypes as C
import os

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
# libocfd_gpu.so: --fmad=false build (every multiply and add rounded separately, bit-identical to
# the CPU restatement where no transcendental enters); OCFD_B200_LIB=fma selects
# libocfd_gpu_fma.so, the same sources with contracted multiply-adds
VARIANT = os.environ.get("OCFD_B200_LIB", "exact")
if VARIANT not in ("exact", "fma"):
    raise ValueError("OCFD_B200_LIB must be 'exact' or 'fma'")
LIBPATH = os.path.join(HERE, "libocfd_gpu_fma.so" if VARIANT == "fma" else "libocfd_gpu.so")

_lib = None


class OcfdError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("OpenCFD-Comb GPU error %d: %s" % (code, msg))
        self.code = code


def lib():
    """Loads libocfd_gpu.so (built by `make -C opencfd-comb_b200`)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise OcfdError(abi.ERR_CUDA, "%s is not built (run make -C opencfd-comb_b200%s)" %
                            (os.path.basename(LIBPATH), " fma" if VARIANT == "fma" else ""))
        L = C.CDLL(LIBPATH)
        for name, (res, args) in abi.GPU_SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _chk(rc):
    if rc != 0:
        raise OcfdError(rc, lib().ocfd_gpu_last_error().decode())


class Solver:
    """One grid, one GPU, one stream (the reference's single MPI rank)."""

    def __init__(self, case, metrics=None):
        L = lib()
        self.case = case
        bc = case.bcdata()
        _chk(L.ocfd_gpu_init(C.byref(case.params), C.byref(case.thermo),
                             C.byref(case.kin) if case.kin is not None else None, C.byref(case.trans),
                             C.byref(bc) if bc is not None else None, abi.dptr(case.coords), abi.dptr(metrics)))
        self.tt = 0.0
        self.istep = 0

    # ---- start-up (OCFD_NS_Solver.f90:15-18) ----
    def init_state(self, tt=0.0):
        c = self.case
        _chk(lib().ocfd_gpu_init_state(abi.dptr(c.prim5), abi.dptr(c.di), tt))
        self.tt = tt

    def upload_state(self, f, di, prims):
        _chk(lib().ocfd_gpu_upload_state(abi.dptr(f), abi.dptr(di), abi.dptr(prims)))

    # ---- the hot path ----
    def flow_time_advance(self, dt1, tt=None):
        _chk(lib().ocfd_gpu_flow_advance(dt1, self.tt if tt is None else tt))

    def chemical_time_advance(self, dt2, nsub=1):
        """nsub x Chemical_time_advance(dt2) followed by comput_T_P."""
        _chk(lib().ocfd_gpu_chem_advance(dt2, nsub))

    def step(self, dt, if_reaction=0, nsub=1):
        """One NS_solver time step (OCFD_NS_Solver.f90:28-46) as a replayed CUDA graph."""
        _chk(lib().ocfd_gpu_step(dt, self.tt, if_reaction, nsub))
        self.istep += 1
        self.tt += dt

    def run(self, dt, nsteps, if_reaction=0, nsub=1):
        """nsteps steps back to back (NS_solver's loop without I/O steps): chunks of 16 steps are
        one graph launch each, the wall-disturbance time of every step is picked on the device."""
        _chk(lib().ocfd_gpu_run(dt, self.tt, nsteps, if_reaction, nsub))
        self.istep += nsteps
        for _ in range(nsteps):
            self.tt += dt

    def show_flow_msg(self):
        """Mean total energy and kinetic energy (OCFD_Time_Adv.f90:210-223)."""
        e, k = C.c_double(), C.c_double()
        _chk(lib().ocfd_gpu_diag(C.byref(e), C.byref(k)))
        return e.value, k.value

    # ---- state transfer ----
    def download_state(self):
        c = self.case
        nx, ny, nz = c.shape
        hs = c.halo_shape()
        f = np.empty((5, nz, ny, nx))
        di = np.empty((c.params.n_spec,) + hs)
        prims = np.empty((7,) + hs)
        _chk(lib().ocfd_gpu_download_state(abi.dptr(f), abi.dptr(di), abi.dptr(prims)))
        return f, di, prims

    def rhybrid(self):
        r = np.empty(self.case.halo_shape())
        _chk(lib().ocfd_gpu_download_rhybrid(abi.dptr(r)))
        return r

    def metrics(self):
        m = np.empty((10,) + self.case.halo_shape())
        _chk(lib().ocfd_gpu_download_metrics(abi.dptr(m)))
        return m

    def stats(self):
        a, b = C.c_longlong(), C.c_longlong()
        _chk(lib().ocfd_gpu_stats(C.byref(a), C.byref(b)))
        return a.value, b.value

    # ---- save / show without a host sync (save_flow_data, show_flow_msg) ----
    def diag_begin(self):
        _chk(lib().ocfd_gpu_diag_begin())

    def diag_end(self):
        e, k = C.c_double(), C.c_double()
        _chk(lib().ocfd_gpu_diag_end(C.byref(e), C.byref(k)))
        return e.value, k.value

    def snapshot(self, istep, tt):
        _chk(lib().ocfd_gpu_snapshot(istep, tt))

    def snapshot_wait(self):
        """(Istep, tt, view of the pinned (5 + Ns, nz, ny, nx) buffer); the view is valid until
        the second-next snapshot and while the solver is open."""
        nx, ny, nz = self.case.shape
        nf = 5 + self.case.params.n_spec
        ist, t, ptr = C.c_int(), C.c_double(), C.POINTER(C.c_double)()
        _chk(lib().ocfd_gpu_snapshot_wait(C.byref(ist), C.byref(t), C.byref(ptr)))
        return ist.value, t.value, np.ctypeslib.as_array(ptr, shape=(nf, nz, ny, nx))

    def save_flow_data_async(self, path, istep, tt):
        """save_flow_data (OCFD_IO.f90:39-64) overlapped with the following steps: the device
        packs the fields and copies them to pinned memory on a copy stream; the previous save is
        collected here (its copy long finished) and written to disk by a background thread that
        touches only that pinned buffer. flush_saves() completes everything."""
        import threading
        from . import files
        if not hasattr(self, "_saves"):
            self._saves, self._writers = [], []
        if len(self._saves) == 1:
            self._collect()
        while len(self._writers) > 1:  # the slot about to be reused must be written out
            self._writers.pop(0).join()
        self.snapshot(istep, tt)
        self._saves.append(path)
        self._files = files
        self._threading = threading

    def _collect(self):
        path = self._saves.pop(0)
        ist, t, a = self.snapshot_wait()
        w = self._threading.Thread(target=self._files.write_flow_data, args=(path, ist, t, a))
        w.start()
        self._writers.append(w)

    def flush_saves(self):
        while getattr(self, "_saves", []):
            self._collect()
        for w in getattr(self, "_writers", []):
            w.join()
        self._writers = []

    # ---- filtering and analysis (code/others/OCFD_filtering.f90, OCFD_ANA.f90) ----
    def filtering(self, istep, table, nfiltering):
        """filtering after step istep (OCFD_NS_Solver.f90:48); table from post.filter_table.
        Returns 1 when a filter group ran."""
        t = np.ascontiguousarray(table, dtype=np.float64)
        applied = C.c_int()
        _chk(lib().ocfd_gpu_filtering(istep, nfiltering, abi.dptr(t), C.byref(applied)))
        return applied.value

    def keep_viscosity(self, on=True):
        _chk(lib().ocfd_gpu_keep_viscosity(1 if on else 0))

    def ana_box(self, tt=None):
        out = np.empty(19)
        _chk(lib().ocfd_gpu_ana_box(self.tt if tt is None else tt, abi.dptr(out)))
        return out

    def ana_q(self):
        nx, ny, nz = self.case.shape
        q = np.empty((nz, ny, nx))
        _chk(lib().ocfd_gpu_ana_q(abi.dptr(q)))
        return q

    def ana_time_average(self, dt):
        k, t = C.c_int(), C.c_double()
        _chk(lib().ocfd_gpu_ana_time_average(dt, C.byref(k), C.byref(t)))
        return k.value, t.value

    def ana_average(self, upload=None):
        """Downloads (fields, K_average, t_average); upload=(fields, K, t) restores them."""
        nx, ny, nz = self.case.shape
        nf = 5 + self.case.params.n_spec
        if upload is not None:
            f = np.ascontiguousarray(upload[0], dtype=np.float64).reshape(nf, nz, ny, nx)
            k, t = C.c_int(int(upload[1])), C.c_double(float(upload[2]))
            _chk(lib().ocfd_gpu_ana_average(1, abi.dptr(f), C.byref(k), C.byref(t)))
            return None
        a = np.empty((nf, nz, ny, nx))
        k, t = C.c_int(), C.c_double()
        _chk(lib().ocfd_gpu_ana_average(0, abi.dptr(a), C.byref(k), C.byref(t)))
        return a, k.value, t.value

    # ---- stencil tiles ----
    def autotune(self, reps=5):
        """Times the candidate tile shapes on the current state and applies the fastest; returns
        (choice, ms per launch of each candidate)."""
        ch = (C.c_int * 9)()
        ms = (C.c_double * 27)()
        _chk(lib().ocfd_gpu_autotune(reps, ch, ms))
        return list(ch), list(ms)

    def set_tiles(self, choice):
        """choice: 9 ints (see ocfd_gpu_autotune); a shorter choice keeps the computed metric
        form and the stream switches of the defaults (choice[8] = 3: both side streams)."""
        choice = list(choice) + [0, 0, 0, 3][len(choice) - 5:] if len(choice) < 9 else list(choice)
        ch = (C.c_int * 9)(*choice)
        _chk(lib().ocfd_gpu_set_tiles(ch))

    def tiles(self):
        ch = (C.c_int * 9)()
        _chk(lib().ocfd_gpu_get_tiles(ch))
        return list(ch)

    # ---- measurement helpers ----
    @staticmethod
    def profile(enable):
        lib().ocfd_gpu_profile(1 if enable else 0)

    @staticmethod
    def profile_read():
        L = lib()
        out = {}
        for c in range(L.ocfd_gpu_profile_nclass()):
            ms, n = C.c_double(), C.c_longlong()
            L.ocfd_gpu_profile_read(c, C.byref(ms), C.byref(n))
            out[L.ocfd_gpu_profile_name(c).decode()] = (ms.value, n.value)
        return out

    @staticmethod
    def stream():
        return lib().ocfd_gpu_stream()

    @staticmethod
    def launch_count():
        return lib().ocfd_gpu_launch_count()

    def close(self):
        self.flush_saves()
        lib().ocfd_gpu_finalize()


def chem_setup(thermo, kin, realgas=1, timeadv=abi.CHEM_IMPLICIT, const_p=False):
    """Chemistry tables for the batched reactors; const_p: constant-pressure reactors (an extension,
    ocfd_gpu_chem_constant_pressure) instead of the reference's constant-volume one."""
    _chk(lib().ocfd_gpu_chem_setup(C.byref(thermo), C.byref(kin), realgas, timeadv))
    if const_p:
        _chk(lib().ocfd_gpu_chem_constant_pressure(1))


def chem_batch(di, e, dt, nsub=None):
    """Batched 0-D reactors (host arrays, updated in place): di (n, Ns), e (n), dt (n), nsub (n) int32."""
    _chk(lib().ocfd_gpu_chem_batch(len(e), abi.dptr(di), abi.dptr(e), abi.dptr(dt), abi.iptr(nsub)))


def chem_batch_device(n, di_ptr, e_ptr, dt_ptr, nsub_ptr):
    """Same on device pointers (e.g. torch tensors' data_ptr())."""
    _chk(lib().ocfd_gpu_chem_batch_device(n, di_ptr, e_ptr, dt_ptr, nsub_ptr))


def fp64_peak_gflops():
    return lib().ocfd_gpu_fp64_peak_gflops()
