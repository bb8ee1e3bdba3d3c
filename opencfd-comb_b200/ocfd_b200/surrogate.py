"""Learned chemistry surrogate over the library's C ABI (no counterpart in the reference).

The network maps a 0-D reactor state (T, log p, Y_k, log dt) to its increments (dY_k, dT) over dt.
It is trained on the GPU by the library's own tensor-core kernels on states that the FP64 implicit
integrator produced, and it is applied behind a gate: the composition change is projected so that
element and total mass are conserved exactly, the energy follows the reference's formation-enthalpy
bookkeeping, T comes from the conserved energy, and a reactor whose network temperature disagrees
with that T by more than tol_T (or whose composition goes negative, or whose state lies outside the
training range) is advanced by the FP64 integrator instead.
"""
import ctypes as C
import re

import numpy as np

from . import abi, cases, solver

ELEMENT_MASS = {"H": 1.00794e-3, "O": 15.9994e-3, "N": 14.0067e-3, "C": 12.0107e-3, "AR": 39.948e-3,
                "HE": 4.002602e-3}


def composition(name):
    """Atoms per molecule of a species name such as H2O2 or HO2."""
    out = {}
    for el, cnt in re.findall(r"(AR|HE|[A-Z])(\d*)", name.upper()):
        out[el] = out.get(el, 0) + (int(cnt) if cnt else 1)
    return out


def element_projection(names, mi):
    """P = I - G^T (G G^T)^-1 G, G(e, k) = a_ek M_e / M_k: dY -> P dY keeps every element's mass
    fraction (and so the total mass) unchanged."""
    comps = [composition(n) for n in names]
    els = sorted({e for c in comps for e in c})
    G = np.array([[c.get(e, 0) * ELEMENT_MASS[e] / mi[k] for k, c in enumerate(comps)] for e in els])
    return np.eye(len(names)) - G.T @ np.linalg.solve(G @ G.T, G), G


def _dev(torch, a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a)).to("cuda")
    return t if dtype is None else t.to(dtype)


class Surrogate:
    """Training and evaluation driver (device buffers through torch, kernels through the C ABI)."""

    def __init__(self):
        import torch
        self.torch = torch
        self.L = solver.lib()
        self.names, self.th, self.kin, _ = cases.h2air_structs()
        self.ns = len(self.names)
        solver.chem_setup(self.th, self.kin, 1, abi.CHEM_IMPLICIT)
        self.mi = np.array([self.th.mi[k] for k in range(self.ns)])
        self.proj, self.G = element_projection(self.names, self.mi)

    def reactors(self, n, seed):
        names, th, kin, di, E, dt, nsub, T = cases.reactors(n=n, seed=seed)
        return di, E, dt, nsub

    def fp64(self, di, E, dt, nsub):
        """FP64 implicit integration on the GPU (device tensors in, updated copies out)."""
        t = self.torch
        # fresh copies (synchronous host-to-device), not clones: the library runs on its own stream
        d_di, d_e = _dev(t, di), _dev(t, E)
        d_dt, d_ns = _dev(t, dt), _dev(t, nsub)
        solver.chem_batch_device(len(E), d_di.data_ptr(), d_e.data_ptr(), d_dt.data_ptr(), d_ns.data_ptr())
        return d_di, d_e

    def temperature(self, d_di, d_e):
        T = self.torch.empty(d_e.shape[0], dtype=self.torch.float64, device="cuda")
        solver._chk(self.L.ocfd_gpu_chem_temperature(d_e.shape[0], d_di.data_ptr(), d_e.data_ptr(), T.data_ptr()))
        return T

    def train(self, n=1 << 18, epochs=30, batch=1024, lr=2e-3, seed=0):
        di, E, dt, nsub = self.reactors(n, seed)
        t = self.torch
        d_di0, d_e0, d_dt = _dev(t, di), _dev(t, E), _dev(t, dt)
        d_di1, d_e1 = self.fp64(di, E, dt, nsub)
        hist = np.zeros(epochs)
        P = np.ascontiguousarray(self.proj)
        solver._chk(self.L.ocfd_gpu_surrogate_train(n, d_di0.data_ptr(), d_e0.data_ptr(), d_dt.data_ptr(),
                                                    d_di1.data_ptr(), d_e1.data_ptr(), abi.dptr(P), epochs, batch,
                                                    lr, seed, abi.dptr(hist)))
        return hist

    def flow_samples(self, case, nsteps, n_sample, seed=0):
        """Cell states of a reacting flow after nsteps FP64 steps (a snapshot of the run), as
        reactors with the step's chemistry time and sub-step count."""
        g = solver.Solver(case)
        g.init_state()
        for s in range(nsteps):
            g.tt = s * case.dt
            g.step(case.dt, 1, case.nsub)
        f, di, prims = g.download_state()
        g.close()
        return self.samples_from_state(case, di, prims, n_sample, seed)

    def samples_from_state(self, case, di, prims, n_sample, seed=0):
        """n_sample cells (seeded choice without replacement) of a downloaded flow state (di and
        the primitives as ocfd_gpu_download_state writes them) as reactors (densities, energy,
        chemistry time, sub-steps)."""
        L4 = 4
        dii = di[:, L4:-L4, L4:-L4, L4:-L4].reshape(self.ns, -1).T
        E = prims[6][L4:-L4, L4:-L4, L4:-L4].reshape(-1)
        rng = np.random.default_rng(seed)
        idx = rng.choice(len(E), size=min(n_sample, len(E)), replace=False)
        n = len(idx)
        return (np.ascontiguousarray(dii[idx]), np.ascontiguousarray(E[idx]), np.full(n, case.dt),
                np.full(n, case.nsub, dtype=np.int32))

    def c4_states(self, n_reactors=1 << 22, jet_cells=1 << 21, seed=0, jet_shape=(384, 256, 256)):
        """The learned-chemistry state set: C3 reactors (seeded draws: T 900-2200 K, equivalence ratio
        0.3-3, product fraction 0-0.5, dt log-uniform in 1e-8..1e-6 s, 1 atm) at two points of their
        trajectory (the draw and the state after one FP64 constant-pressure integration over dt),
        plus cells of two FP64 snapshots of the reacting jet (after 8 and 16 steps). With the
        defaults: 2 x 2^22 reactor states + 2^21 jet cells = 10 x 2^20 states. Returns
        (di, E, dt, nsub, source) with source 0 = reactor, 1 = jet."""
        di, E, dt, nsub = self.reactors(n_reactors, seed)
        solver.chem_setup(self.th, self.kin, 1, abi.CHEM_IMPLICIT, const_p=True)
        d1, e1 = self.fp64(di, E, dt, nsub)
        solver.chem_setup(self.th, self.kin, 1, abi.CHEM_IMPLICIT)
        parts = [(di, E, dt, nsub), (d1.cpu().numpy(), e1.cpu().numpy(), dt, nsub)]
        del d1, e1
        case = cases.jet(*jet_shape)
        g = solver.Solver(case)
        g.init_state()
        L = solver.lib()
        for s0, s1, sd in ((0, 8, seed + 1), (8, 16, seed + 2)):
            solver._chk(L.ocfd_gpu_run(case.dt, s0 * case.dt, s1 - s0, 1, case.nsub))
            _, dj, pj = g.download_state()
            parts.append(self.samples_from_state(case, dj, pj, jet_cells // 2, sd))
            del dj, pj
        g.close()
        solver.chem_setup(self.th, self.kin, 1, abi.CHEM_IMPLICIT)
        src = np.concatenate([np.full(len(p[1]), 0 if k < 2 else 1, np.int8) for k, p in enumerate(parts)])
        return (np.concatenate([p[0] for p in parts]), np.concatenate([p[1] for p in parts]),
                np.concatenate([p[2] for p in parts]), np.concatenate([p[3] for p in parts]).astype(np.int32), src)

    @staticmethod
    def split(n, n_hold, seed=0):
        """Seeded split of n states into (train index, held-out index) with n_hold held out."""
        perm = np.random.default_rng(seed).permutation(n)
        return np.sort(perm[n_hold:]), np.sort(perm[:n_hold])

    def train_on(self, parts, epochs=20, batch=1024, lr=2e-3, seed=0):
        """Trains on the concatenation of (di, E, dt, nsub) reactor sets, targets from the FP64
        integrator."""
        t = self.torch
        di = np.concatenate([p[0] for p in parts])
        E = np.concatenate([p[1] for p in parts])
        dt = np.concatenate([p[2] for p in parts])
        nsub = np.concatenate([p[3] for p in parts]).astype(np.int32)
        n = (len(E) // batch) * batch
        di, E, dt, nsub = di[:n], E[:n], dt[:n], nsub[:n]
        solver.chem_setup(self.th, self.kin, 1, abi.CHEM_IMPLICIT)
        d_di0, d_e0, d_dt = _dev(t, di), _dev(t, E), _dev(t, dt)
        d_di1, d_e1 = self.fp64(di, E, dt, nsub)
        hist = np.zeros(epochs)
        P = np.ascontiguousarray(self.proj)
        solver._chk(self.L.ocfd_gpu_surrogate_train(n, d_di0.data_ptr(), d_e0.data_ptr(), d_dt.data_ptr(),
                                                    d_di1.data_ptr(), d_e1.data_ptr(), abi.dptr(P), epochs, batch,
                                                    lr, seed, abi.dptr(hist)))
        return hist

    def evaluate(self, n=1 << 16, seed=12345, tol_T=5.0):
        """Held-out reactors: errors of the ungated network and of the gated surrogate against the
        FP64 integrator, the fallback fraction and the element-conservation residual."""
        di, E, dt, nsub = self.reactors(n, seed)
        return self.evaluate_on(di, E, dt, nsub, tol_T)

    def evaluate_on(self, di, E, dt, nsub, tol_T=5.0):
        """The same on given states (di (n, Ns), E, dt, nsub)."""
        t = self.torch
        n = len(E)
        d_di, d_e, d_dt, d_ns = _dev(t, di), _dev(t, E), _dev(t, dt), _dev(t, nsub)
        f_di, f_e = self.fp64(di, E, dt, nsub)
        T_ref = self.temperature(f_di, f_e)
        o_di = t.empty_like(d_di)
        o_e, Tp, Te = t.empty_like(d_e), t.empty_like(d_e), t.empty_like(d_e)
        t.cuda.synchronize()
        solver._chk(self.L.ocfd_gpu_surrogate_predict(n, d_di.data_ptr(), d_e.data_ptr(), d_dt.data_ptr(),
                                                      o_di.data_ptr(), o_e.data_ptr(), Tp.data_ptr(), Te.data_ptr()))
        g_di, g_e = _dev(t, di), _dev(t, E)
        nfb = C.c_int()
        solver._chk(self.L.ocfd_gpu_chem_batch_surrogate(n, g_di.data_ptr(), g_e.data_ptr(), d_dt.data_ptr(),
                                                         d_ns.data_ptr(), tol_T, C.byref(nfb)))
        T_g = self.temperature(g_di, g_e)
        T0 = self.temperature(d_di, d_e)

        def Y(x):
            x = x.cpu().numpy()
            return x / x.sum(axis=1, keepdims=True)

        Yr, Yn, Yg, Y0 = Y(f_di), Y(o_di), Y(g_di), Y(d_di)
        Tr = T_ref.cpu().numpy()
        el0 = Y0 @ self.G.T
        return {
            "n": n,
            "fallback_fraction": nfb.value / n,
            "ungated_T_err_max_K": float(np.abs(Te.cpu().numpy() - Tr).max()),
            "ungated_T_err_rel_max": float((np.abs(Te.cpu().numpy() - Tr) / Tr).max()),
            "ungated_Y_err_max": float(np.abs(Yn - Yr).max()),
            "gated_T_err_max_K": float(np.abs(T_g.cpu().numpy() - Tr).max()),
            "gated_T_err_rel_max": float((np.abs(T_g.cpu().numpy() - Tr) / Tr).max()),
            "gated_Y_err_max": float(np.abs(Yg - Yr).max()),
            "no_reaction_T_err_max_K": float(np.abs(T0.cpu().numpy() - Tr).max()),
            "no_reaction_Y_err_max": float(np.abs(Y0 - Yr).max()),
            "element_residual_max": float(np.abs(Yg @ self.G.T - el0).max()),
        }

    def blob(self):
        n = self.L.ocfd_gpu_surrogate_blob(None, 0, 0)
        buf = (C.c_float * n)()
        rc = self.L.ocfd_gpu_surrogate_blob(buf, n, 0)
        if rc != 0:
            raise solver.OcfdError(rc, "surrogate blob")
        return np.frombuffer(buf, dtype=np.float32).copy()

    def load(self, blob):
        b = np.ascontiguousarray(blob, dtype=np.float32)
        rc = self.L.ocfd_gpu_surrogate_blob(b.ctypes.data_as(C.POINTER(C.c_float)), len(b), 1)
        if rc != 0:
            raise solver.OcfdError(rc, "surrogate blob")
