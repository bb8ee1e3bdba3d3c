"""Seeded synthetic workloads with the shapes of the OpenCFD-Comb benchmark configurations.

No dataset or restart file of the reference is available on the GPU box, so every workload is
generated here from a fixed NumPy seed:

  isotropic(n)      decaying compressible isotropic turbulence, 64^3 periodic box of side
                    2*pi*1e-3 m, air as one perfect-gas species (gamma = 1.4), Pr = 0.7,
                    Sutherland viscosity, WENO5 + CD6, Steger-Warming; solenoidal random-phase
                    velocity with E(k) ~ k^4 exp(-2 (k/k0)^2), k0 = 4, M_t = 0.3, Re_lambda = 70
                    (construction as cases/isotropic/init-isotropic.f90, numpy FFT instead of
                    the Fortran FFT); dt from CFL 0.5 on the initial field.
  flatplate(...)    Mach 2.25 flat-plate boundary layer, 1024x160x128, x uniform, y tanh-stretched,
                    z periodic; T_inf = 169.4 K, Re = 635000/inch; compressible similarity inflow
                    profile (Blasius + Crocco-Busemann, Howarth-Dorodnitsyn stretching); isothermal
                    wall at the adiabatic-wall temperature; Rai blowing/suction strip of amplitude
                    0.01 U_inf with 8 spanwise x 8 temporal modes from a seeded phase table;
                    HYBRID (UD7L / WENO7 / WENO5, pressure sensor 1) or OMP6.
  reactors(n)       2^20 H2-air 0-D reactors, 9 species: T ~ U(900, 2200) K, equivalence ratio
                    ~ U(0.3, 3.0), product fraction ~ U(0, 0.5), p = 1 atm, dt ~ logU(1e-8, 1e-6) s.

Arrays use the reference's Fortran layout: a halo array (1-LAP:nx+LAP, ...) is a numpy array of
shape (nz+2L, ny+2L, nx+2L); an interior array is (nz, ny, nx); f is (5, nz, ny, nx).
"""
import ctypes as C
import json
import math
import os

import numpy as np

from . import abi

LAP = 4
R0 = 8.314
ATM = 1.013e5
DATA = os.path.join(os.path.dirname(__file__), "data", "h2_air_9sp.json")


class Case:
    """Everything one solver run needs: the ABI structs, grid, and initial primitives."""

    def __init__(self, name):
        self.name = name
        self.params = abi.Params()
        self.thermo = abi.Thermo()
        self.kin = None
        self.trans = abi.Transport()
        self.bc = None          # dict of numpy arrays for abi.BcData
        self.coords = None      # (3, HZ, HY, HX)
        self.prim5 = None       # (5, nz, ny, nx): d, u, v, w, T  (read_flow_data content)
        self.di = None          # (Ns, nz, ny, nx)
        self.dt = 0.0
        self.nsteps = 1
        self.if_reaction = 0
        self.nsub = 1
        self.filters = []    # filter groups (post.filter_table), applied after every step
        self.analysis = []   # analysis entries (post.ana_table), OCFD_analysis after every step

    @property
    def shape(self):
        p = self.params
        return p.nx, p.ny, p.nz

    @property
    def ncell(self):
        return self.params.nx * self.params.ny * self.params.nz

    def halo_shape(self):
        p = self.params
        return (p.nz + 2 * LAP, p.ny + 2 * LAP, p.nx + 2 * LAP)

    def save(self, path):
        """Writes the case file read by the compiled host driver (host/ns_solver.cpp): the ABI
        records as bytes, then dt / nsteps / chemistry switch / sub-steps, grid, initial
        primitives, species densities, the boundary tables, and the filter and analysis tables
        (Para%Filter, Para%ANA_Para)."""
        import struct
        with open(path, "wb") as fh:
            fh.write(b"OCFDCASE")
            fh.write(struct.pack("<5i", 2, C.sizeof(abi.Params), C.sizeof(abi.Thermo), C.sizeof(abi.Kinetics),
                                 C.sizeof(abi.Transport)))
            fh.write(bytes(self.params))
            fh.write(bytes(self.thermo))
            fh.write(struct.pack("<i", 1 if self.kin is not None else 0))
            if self.kin is not None:
                fh.write(bytes(self.kin))
            fh.write(bytes(self.trans))
            fh.write(struct.pack("<d3i", self.dt, self.nsteps, self.if_reaction, self.nsub))
            coords = np.ascontiguousarray(self.coords, dtype=np.float64)
            fh.write(struct.pack("<q", coords.size // 3))
            fh.write(coords.tobytes())
            prim = np.ascontiguousarray(self.prim5, dtype=np.float64)
            fh.write(struct.pack("<q", prim.size // 5))
            fh.write(prim.tobytes())
            di = np.ascontiguousarray(self.di, dtype=np.float64)
            fh.write(struct.pack("<i", self.params.n_spec))
            fh.write(di.tobytes())
            fh.write(struct.pack("<i", 1 if self.bc is not None else 0))
            if self.bc is not None:
                for key in ("inlet", "upper", "wall_pertb", "tm", "fait"):
                    a = self.bc.get(key)
                    a = np.zeros(0) if a is None else np.ascontiguousarray(a, dtype=np.float64).ravel()
                    fh.write(struct.pack("<q", a.size))
                    fh.write(a.tobytes())
            from . import post
            ft, nf = post.filter_table(self.filters)
            at, na = post.ana_table(self.analysis)
            fh.write(struct.pack("<i", nf))
            fh.write(np.ascontiguousarray(ft).tobytes())
            fh.write(struct.pack("<i", na))
            fh.write(np.ascontiguousarray(at).tobytes())

    def bcdata(self):
        """abi.BcData pointing at this case's arrays (kept alive by the case)."""
        if self.bc is None:
            return None
        b = abi.BcData()
        b.inlet = abi.dptr(self.bc["inlet"])
        b.upper = abi.dptr(self.bc["upper"])
        b.wall_pertb = abi.dptr(self.bc["wall_pertb"])
        b.n_tm = len(self.bc["tm"])
        b.tm = abi.dptr(self.bc["tm"])
        b.fait = abi.dptr(self.bc["fait"])
        return b


# ---------------------------------------------------------------- species / mechanism data

def load_mechanism():
    with open(DATA) as fh:
        return json.load(fh)


def thermo_struct(species, n_tct, tct, tct_max):
    th = abi.Thermo()
    th.n_spec = len(species)
    th.n_tct = n_tct
    for j, t in enumerate(tct):
        th.tct[j] = t
    th.tct_max = tct_max
    for k, s in enumerate(species):
        th.mi[k] = s["mi"]
        th.spec_flag[k] = s["spec_flag"]
        for j in range(n_tct):
            for c in range(7):
                th.coef[k][j][c] = s["coef"][j][c]
    return th


def air_thermo():
    """One 'AIR' species (Mi = 0.029 kg/mol, cases/M2.25_air/specie-air.in) for IF_RealGas = 0,
    where only R = R0/Mi enters (Cv = 2.5 R, CHEM_thermdyn.f90:114-168)."""
    sp = [dict(name="AIR", mi=0.029, spec_flag=2, coef=[[3.5, 0, 0, 0, 0, 0, 0]])]
    return thermo_struct(sp, 1, [], 5000.0)


def h2air_structs():
    mech = load_mechanism()
    th = mech["thermo"]
    thermo = thermo_struct(th["species"], th["n_tct"], th["tct"], th["tct_max"])
    rc = mech["kinetics"]
    kin = abi.Kinetics()
    kin.n_spec = rc["n_spec"]
    kin.n_reac = rc["n_reac"]
    kin.rereac = rc["rereac"]
    for j, r in enumerate(rc["reactions"]):
        kin.af_type[j] = r["af_type"]
        kin.tr_reac[j] = r["tr_reac"]
        kin.fc_troe[j] = r["fc_troe"]
        for s in range(2):
            kin.af[j][s], kin.bf[j][s], kin.ef[j][s] = r["arr"][s]
        kin.ar[j], kin.br[j], kin.er[j] = r["rev"]
        for c in range(5):
            kin.park[j][c] = r["park"][c]
        for i in range(rc["n_spec"]):
            kin.vf[j][i] = r["vf"][i]
            kin.vr[j][i] = r["vr"][i]
            kin.treff[j][i] = r["treff"][i]
    names = [s["name"] for s in th["species"]]
    tr = abi.Transport()
    tr.flag_vis = tr.flag_cond = tr.flag_diff = 1
    tr.amu0, tr.pr, tr.sc = 1.789e-5, 0.7, 1.0
    for k, n in enumerate(names):
        for c in range(4):
            tr.mu_an[k][c] = mech["viscosity"][n][c]
            tr.k_an[k][c] = mech["conductivity"][n][c]
    for a, b, v in mech["diffusion"]:
        ia, ib = names.index(a), names.index(b)
        for c in range(4):
            tr.d_an[ia][ib][c] = v[c]
            tr.d_an[ib][ia][c] = v[c]
    return names, thermo, kin, tr


def energy_realgas(thermo, di, T):
    """comput_E_rgas (CHEM_thermdyn.f90:203-231) in numpy, for building initial states.
    di: (Ns, ...) species densities; T: (...)."""
    ns, nt = thermo.n_spec, thermo.n_tct
    coef = np.array([[list(thermo.coef[k][j]) for j in range(nt)] for k in range(ns)])  # (ns, nt, 7)
    tct = [thermo.tct[j] for j in range(nt - 1)]
    ri = np.array([R0 / thermo.mi[k] for k in range(ns)])
    ect = np.zeros((ns, nt))
    for j in range(nt - 1):
        t = tct[j]
        d = coef[:, j + 1] - coef[:, j]
        ect[:, j + 1] = -(d[:, 0] * t + d[:, 1] * t ** 2 / 2 + d[:, 2] * t ** 3 / 3 + d[:, 3] * t ** 4 / 4
                          + d[:, 4] * t ** 5 / 5) + ect[:, j]
    jc = np.zeros(T.shape, dtype=int)
    for j in range(nt - 1):
        jc = np.where(T > tct[j], j + 1, jc)
    Tm = np.minimum(T, thermo.tct_max)
    w = ri.reshape((ns,) + (1,) * T.ndim) * di
    c = coef[:, jc]  # (ns, ..., 7)
    e_sub = ((c[..., 0] - 1.0) * Tm + c[..., 1] * Tm ** 2 / 2 + c[..., 2] * Tm ** 3 / 3 + c[..., 3] * Tm ** 4 / 4
             + c[..., 4] * Tm ** 5 / 5 + ect[np.arange(ns).reshape((ns,) + (1,) * T.ndim), jc])
    cv_max = (c[..., 0] - 1.0) + c[..., 1] * Tm + c[..., 2] * Tm ** 2 + c[..., 3] * Tm ** 3 + c[..., 4] * Tm ** 4
    e_k = e_sub + np.where(T > thermo.tct_max, cv_max * (T - thermo.tct_max), 0.0)
    return (w * e_k).sum(axis=0)


# ---------------------------------------------------------------- common parameter setup

def base_params(nx, ny, nz, ns):
    p = abi.Params()
    p.nx, p.ny, p.nz, p.lap, p.n_spec = nx, ny, nz, LAP, ns
    p.scheme_invis = abi.SCHEME_WENO5
    p.scheme_vis = abi.SCHEME_CD6
    p.if_viscous = 1
    p.flux_splitting = abi.SPLIT_SW
    p.ibc = abi.BC_NONE
    p.ud7l_diss = 1.0
    for m in range(100):
        p.hybrid_para[m] = 1.0
    p.if_realgas = 0
    p.chem_timeadv = abi.CHEM_EULER
    p.istep_show = 1
    return p


def coords_1d(x, y, z):
    """read_mesh1d (OCFD_mesh.f90:218-249): Axx(i,j,k)=x(i) etc. on the interior; halo = 1.0
    (allocate_flow_data's initial value)."""
    nx, ny, nz = len(x), len(y), len(z)
    c = np.ones((3, nz + 2 * LAP, ny + 2 * LAP, nx + 2 * LAP))
    sl = (slice(LAP, LAP + nz), slice(LAP, LAP + ny), slice(LAP, LAP + nx))
    c[0][sl] = np.broadcast_to(x[None, None, :], (nz, ny, nx))
    c[1][sl] = np.broadcast_to(y[None, :, None], (nz, ny, nx))
    c[2][sl] = np.broadcast_to(z[:, None, None], (nz, ny, nx))
    return c


def sutherland(T, amu0=1.789e-5):
    return amu0 * np.sqrt((T / 288.15) ** 3) * (288.15 + 110.4) / (110.4 + T)


# ---------------------------------------------------------------- C1: isotropic turbulence

def species_subset(names_wanted, realgas=1, wilke=False):
    """Thermo (+ transport, kinetics when all nine H2-air species are asked for) for a subset of
    the H2-air species, in the requested order."""
    names, th9, kin9, tr9 = h2air_structs()
    mech = load_mechanism()
    sp = [mech["thermo"]["species"][names.index(n)] for n in names_wanted]
    th = thermo_struct(sp, mech["thermo"]["n_tct"], mech["thermo"]["tct"], mech["thermo"]["tct_max"])
    tr = abi.Transport()
    if wilke:
        tr = tr9 if list(names_wanted) == names else tr9
    tr.amu0, tr.pr, tr.sc = 1.789e-5, 0.7, 1.0
    if not wilke:
        tr.flag_vis = tr.flag_cond = tr.flag_diff = 0
    kin = kin9 if list(names_wanted) == names else None
    return th, tr, kin


def isotropic(n=64, seed=0, k0=4.0, mach_t=0.3, re_lambda=70.0, T0=300.0, cfl=0.5, scheme="WENO5",
              flux_splitting=abi.SPLIT_SW, nsteps=100, species=None, Y=None, wilke=False):
    """species=None: one perfect-gas AIR species; otherwise a list of H2-air species names with
    mass fractions Y, NASA-fit thermodynamics (IF_RealGas=1), Sutherland/Pr/Sc or Wilke transport."""
    ns = 1 if species is None else len(species)
    case = Case("isotropic-%d" % n)
    p = base_params(n, n, n, ns)
    p.scheme_invis = abi.SCHEME_NAMES[scheme]
    p.flux_splitting = flux_splitting
    p.iperiodic[0] = p.iperiodic[1] = p.iperiodic[2] = 1
    L = 2.0 * math.pi * 1.0e-3
    for d in range(3):
        p.periodic_span[d][d] = L
    case.params = p
    if species is None:
        case.thermo = air_thermo()
        tr = abi.Transport()
        tr.flag_vis = tr.flag_cond = tr.flag_diff = 0
        tr.amu0, tr.pr, tr.sc = 1.789e-5, 0.7, 1.0
        case.trans = tr
        Rmix = R0 / 0.029
    else:
        th, tr, kin = species_subset(species, wilke=wilke)
        case.thermo, case.trans, case.kin = th, tr, kin
        p.if_realgas = 1
        p.chem_timeadv = abi.CHEM_IMPLICIT
        Y = np.asarray(Y, dtype=float) / np.sum(Y)
        Rmix = float(sum(Y[k] * R0 / th.mi[k] for k in range(ns)))
    h = L / n
    x = np.arange(n) * h
    case.coords = coords_1d(x, x, x)

    rng = np.random.default_rng(seed)
    kk = np.fft.fftfreq(n) * n
    KZ, KY, KX = np.meshgrid(kk, kk, kk, indexing="ij")
    K2 = KX ** 2 + KY ** 2 + KZ ** 2
    Km = np.sqrt(K2)
    Ek = Km ** 4 * np.exp(-2.0 * (Km / k0) ** 2)
    amp = np.sqrt(np.where(Km > 0, Ek / (4.0 * math.pi * np.maximum(K2, 1e-30)), 0.0))
    a = (rng.standard_normal((3, n, n, n)) + 1j * rng.standard_normal((3, n, n, n)))
    kdota = (KX * a[0] + KY * a[1] + KZ * a[2]) / np.maximum(K2, 1e-30)
    a = np.stack([a[0] - KX * kdota, a[1] - KY * kdota, a[2] - KZ * kdota]) * amp
    vel = np.real(np.fft.ifftn(a, axes=(1, 2, 3)))  # (3, z, y, x) with component order u(x), v(y), w(z)
    vel = np.stack([vel[0], vel[1], vel[2]])
    c0 = math.sqrt(1.4 * Rmix * T0)
    urms = math.sqrt(np.mean(vel[0] ** 2 + vel[1] ** 2 + vel[2] ** 2))
    vel *= mach_t * c0 / urms
    up = math.sqrt(np.mean(vel[0] ** 2 + vel[1] ** 2 + vel[2] ** 2) / 3.0)
    dudx = np.real(np.fft.ifftn(1j * KX * np.fft.fftn(vel[0]) * (2 * math.pi / L)))
    lam = math.sqrt(np.mean(vel[0] ** 2) / np.mean(dudx ** 2))
    mu = float(sutherland(np.array(T0)))
    rho = re_lambda * mu / (up * lam)
    d = np.full((n, n, n), rho)
    T = np.full((n, n, n), T0)
    case.prim5 = np.ascontiguousarray(np.stack([d, vel[0], vel[1], vel[2], T]))
    if species is None:
        case.di = np.ascontiguousarray(d[None].copy())
    else:
        case.di = np.ascontiguousarray(np.stack([d * Y[k] for k in range(ns)]))
    umax = np.max(np.abs(vel[0]) + np.abs(vel[1]) + np.abs(vel[2]))
    case.dt = cfl * h / (umax + c0)
    case.nsteps = nsteps
    case.info = dict(rho=rho, u_prime=up, lambda_taylor=lam, mu=mu, c0=c0, h=h)
    return case


# ---------------------------------------------------------------- C2: M2.25 flat plate

def _blasius(eta_max=12.0, n=4001):
    """f''' + f f'' = 0, f(0)=f'(0)=0, f'(inf)=1 (eta = y sqrt(U/(2 nu x)))."""
    eta = np.linspace(0.0, eta_max, n)
    hstep = eta[1] - eta[0]

    def shoot(s):
        y = np.array([0.0, 0.0, s])
        out = [y.copy()]
        for _ in range(n - 1):
            def fn(v):
                return np.array([v[1], v[2], -v[0] * v[2]])
            k1 = fn(y); k2 = fn(y + 0.5 * hstep * k1); k3 = fn(y + 0.5 * hstep * k2); k4 = fn(y + hstep * k3)
            y = y + hstep / 6.0 * (k1 + 2 * k2 + 2 * k3 + k4)
            out.append(y.copy())
        return np.array(out)

    lo, hi = 0.3, 0.6
    for _ in range(60):
        mid = 0.5 * (lo + hi)
        if shoot(mid)[-1, 1] > 1.0:
            hi = mid
        else:
            lo = mid
    sol = shoot(0.5 * (lo + hi))
    return eta, sol[:, 1]


def flatplate(nx=1024, ny=160, nz=128, scheme="HYBRID", seed=0, nsteps=10, theta=(0.005, 0.02),
              x0=0.05, lx=0.2, ly=0.012, lz=0.004445, y1=3.0e-6):
    case = Case("flatplate-%dx%dx%d-%s" % (nx, ny, nz, scheme))
    p = base_params(nx, ny, nz, 1)
    p.scheme_invis = abi.SCHEME_NAMES[scheme]
    p.iperiodic[2] = 1
    p.periodic_span[2][2] = lz
    p.ibc = abi.BC_BOUNDARYLAYER
    p.hybrid_para[0] = 1.0          # shock sensor 1 (pressure second difference)
    p.hybrid_para[1] = theta[0]
    p.hybrid_para[2] = theta[1]
    p.hybrid_para[3] = 0.0          # no forced patches
    case.params = p
    case.thermo = air_thermo()
    tr = abi.Transport()
    tr.flag_vis = tr.flag_cond = tr.flag_diff = 0
    tr.amu0, tr.pr, tr.sc = 1.789e-5, 0.7, 1.0
    case.trans = tr

    R = R0 / 0.029
    gam = 1.4
    Tinf = 169.4
    M = 2.25
    cinf = math.sqrt(gam * R * Tinf)
    U = M * cinf
    mu_inf = float(sutherland(np.array(Tinf)))
    re_unit = 635000.0 / 0.0254
    rho_inf = re_unit * mu_inf / U
    r = math.sqrt(0.7)
    Taw = Tinf * (1.0 + r * 0.5 * (gam - 1.0) * M * M)
    Tw = Taw

    x = x0 + lx * np.arange(nx) / (nx - 1)
    # tanh stretching with first spacing ~ y1
    s = np.arange(ny) / (ny - 1)
    b = 1.0
    for _ in range(100):
        yy = ly * (1.0 - np.tanh(b * (1.0 - s)) / math.tanh(b))
        if yy[1] > y1:
            b *= 1.05
        else:
            break
    y = ly * (1.0 - np.tanh(b * (1.0 - s)) / math.tanh(b))
    z = lz * np.arange(nz) / nz
    case.coords = coords_1d(x, y, z)

    # similarity profile at the inlet x0
    eta, fp = _blasius()
    T_of_u = lambda uu: Tw + (Taw - Tw) * uu - r * 0.5 * (gam - 1.0) * M * M * Tinf * uu * uu  # noqa: E731
    Tprof = T_of_u(fp)
    nu_inf = mu_inf / rho_inf
    scale = math.sqrt(2.0 * nu_inf * x0 / U)
    yphys = scale * np.concatenate([[0.0], np.cumsum(0.5 * (Tprof[1:] + Tprof[:-1]) / Tinf * np.diff(eta))])
    uin = np.interp(y, yphys, fp, right=1.0) * U
    Tin = np.interp(y, yphys, Tprof, right=Tinf)
    pin = rho_inf * R * Tinf
    din = pin / (R * Tin)
    inlet = np.stack([din, uin, np.zeros(ny), np.zeros(ny), Tin, din])  # [comp][j], di rescaled to d
    upper = np.array([rho_inf, U, 0.0, 0.0, Tinf, rho_inf])

    rng = np.random.default_rng(seed)
    mz = mt = 8
    faiz = rng.random(mz)
    fait = rng.random(mt)
    zl = np.array([1.25 ** (-m) for m in range(mz)])
    zl /= zl.sum()
    tm = np.array([1.25 ** (-m) for m in range(mt)])
    tm /= tm.sum()
    xb, xe = x0 + 0.1 * lx, x0 + 0.2 * lx
    PI = 3.14159265358979
    X, Z = np.meshgrid(x, z)  # (nz, nx)
    seta = 2.0 * PI * (X - xb) / (xe - xb)
    fx = np.where((X >= xb) & (X <= xe), 4.0 / math.sqrt(27.0) * np.sin(seta) * (1.0 - np.cos(seta)), 0.0)
    gz = np.zeros_like(X)
    for m in range(mz):
        gz += zl[m] * np.sin(2.0 * PI * (m + 1) * (Z / lz + faiz[m]))
    wall_pertb = np.ascontiguousarray(fx * gz)  # (nz, nx) = BC%wall_pertb(i,k), i fastest
    freq = 0.1 * U / (xe - xb)
    bcp = [1, 0, 0, 0, Tw, 0.0, 1, 0.01 * U, xb, xe, mt, mz, lz, freq]
    for m, v in enumerate(bcp):
        p.bc_para[m] = v
    case.bc = dict(inlet=np.ascontiguousarray(inlet), upper=upper, wall_pertb=wall_pertb, tm=tm, fait=fait)

    d = np.broadcast_to(din[None, :, None], (nz, ny, nx)).copy()
    u = np.broadcast_to(uin[None, :, None], (nz, ny, nx)).copy()
    T = np.broadcast_to(Tin[None, :, None], (nz, ny, nx)).copy()
    zero = np.zeros((nz, ny, nx))
    case.prim5 = np.ascontiguousarray(np.stack([d, u, zero, zero.copy(), T]))
    case.di = np.ascontiguousarray(d[None].copy())
    dy_min = y[1] - y[0]
    case.dt = 0.5 * min(dy_min / (math.sqrt(gam * R * Tw)), (x[1] - x[0]) / (U + cinf), (z[1] - z[0]) / cinf)
    case.nsteps = nsteps
    case.info = dict(U=U, rho_inf=rho_inf, Tw=Tw, mu_inf=mu_inf, y1=y[1] - y[0])
    return case


# ---------------------------------------------------------------- C3: batched 0-D reactors

def reactors(n=2 ** 20, seed=0, dt_sub_max=1.0e-8, nsub_max=100):
    """Returns (names, thermo, kin, di (n, 9), E (n), dt (n), nsub (n) int32, T (n)).
    nsub: sub-steps per reactor = clamp(ceil(dt / dt_sub_max), 1, nsub_max). The reference uses
    one global Chemical_sub_step; the per-reactor count is this workload's extension."""
    names, thermo, kin, _ = h2air_structs()
    rng = np.random.default_rng(seed)
    T = rng.uniform(900.0, 2200.0, n)
    phi = rng.uniform(0.3, 3.0, n)
    pf = rng.uniform(0.0, 0.5, n)
    dt = np.exp(rng.uniform(math.log(1e-8), math.log(1e-6), n))
    idx = {s: names.index(s) for s in names}
    X = np.zeros((n, len(names)))
    # reactants (mol): 2 phi H2 + O2 + 3.76 N2; complete-combustion products
    react = {"H2": 2 * phi, "O2": np.ones(n), "N2": 3.76 * np.ones(n)}
    prod = {"H2O": np.minimum(2 * phi, 2.0), "H2": np.maximum(2 * phi - 2.0, 0.0), "O2": np.maximum(1.0 - phi, 0.0),
            "N2": 3.76 * np.ones(n)}
    for s, v in react.items():
        X[:, idx[s]] += (1.0 - pf) * v
    for s, v in prod.items():
        X[:, idx[s]] += pf * v
    # trace radicals so that no concentration is exactly zero
    for s in ("O", "OH", "H", "HO2", "H2O2"):
        X[:, idx[s]] += 1e-12
    X /= X.sum(axis=1, keepdims=True)
    mi = np.array([thermo.mi[k] for k in range(len(names))])
    Y = X * mi
    Y /= Y.sum(axis=1, keepdims=True)
    Rmix = (Y * (R0 / mi)).sum(axis=1)
    rho = ATM / (Rmix * T)
    di = np.ascontiguousarray(Y * rho[:, None])
    E = energy_realgas(thermo, di.T.copy(), T)
    nsub = np.clip(np.ceil(dt / dt_sub_max), 1, nsub_max).astype(np.int32)
    return names, thermo, kin, di, np.ascontiguousarray(E), np.ascontiguousarray(dt), nsub, T


# ---------------------------------------------------------------- C5: reacting H2 jet

def _mole_to_mass(names, mi, X):
    X = np.asarray(X, dtype=float)
    X = X / X.sum()
    Y = X * mi
    return Y / Y.sum()


def jet(nx=384, ny=256, nz=256, seed=0, D=1.0e-3, Uj=200.0, Tj=300.0, Uc=10.0, Tc=1100.0, pert=0.02,
        lx_d=30.0, ly_d=10.0, nsteps=200, timeadv=abi.CHEM_IMPLICIT, nsub=1, iflag_inlet=1):
    """Round H2/N2 jet (70/30 by volume, 300 K, 200 m/s, D = 1 mm, tanh-smoothed top hat) into an
    air coflow (1100 K, 10 m/s, 1 atm); x stretched, y/z tanh-clustered toward the jet axis;
    9-species H2-air chemistry, Wilke transport, BC_JET inflow with seeded 2 % velocity noise."""
    names, th, kin, tr = h2air_structs()
    ns = len(names)
    case = Case("jet-%dx%dx%d" % (nx, ny, nz))
    p = base_params(nx, ny, nz, ns)
    p.ibc = abi.BC_JET
    p.bc_para[0] = iflag_inlet
    p.if_realgas = 1
    p.chem_timeadv = timeadv
    case.params = p
    case.thermo, case.kin, case.trans = th, kin, tr
    mi = np.array([th.mi[k] for k in range(ns)])
    Xj = np.zeros(ns); Xj[names.index("H2")] = 0.7; Xj[names.index("N2")] = 0.3
    Xc = np.zeros(ns); Xc[names.index("O2")] = 0.21; Xc[names.index("N2")] = 0.79
    Yj, Yc = _mole_to_mass(names, mi, Xj), _mole_to_mass(names, mi, Xc)
    # grids
    s = np.arange(nx) / (nx - 1)
    x = lx_d * D * (np.expm1(2.0 * s) / np.expm1(2.0))
    def clustered(n, half):
        t = np.linspace(-1.0, 1.0, n)
        b = 1.5
        return half * np.sinh(b * t) / np.sinh(b)
    y = clustered(ny, 0.5 * ly_d * D)
    z = clustered(nz, 0.5 * ly_d * D)
    case.coords = coords_1d(x, y, z)
    # inlet table (BcData_inlet = 2): [comp][k][j]
    Y2, Z2 = np.meshgrid(y, z)  # (nz, ny)
    r = np.sqrt(Y2 ** 2 + Z2 ** 2)
    fr = 0.5 * (1.0 - np.tanh((r - 0.5 * D) / (0.05 * D)))  # 1 in the jet, 0 in the coflow
    rng = np.random.default_rng(seed)
    U = Uc + (Uj - Uc) * fr
    U = U * (1.0 + pert * rng.uniform(-1.0, 1.0, U.shape))
    T = Tc + (Tj - Tc) * fr
    Yk = Yc[:, None, None] + (Yj - Yc)[:, None, None] * fr[None]
    Rmix = (Yk * (R0 / mi)[:, None, None]).sum(axis=0)
    rho = ATM / (Rmix * T)
    inlet = np.zeros((5 + ns, nz, ny))
    inlet[0], inlet[1], inlet[4] = rho, U, T
    inlet[5:] = Yk * rho[None]
    case.bc = dict(inlet=np.ascontiguousarray(inlet), upper=np.zeros(5 + ns), wall_pertb=None, tm=np.zeros(0),
                   fait=np.zeros(0))
    # initial field: the inflow plane extended downstream
    d3 = np.broadcast_to(rho[:, :, None], (nz, ny, nx)).copy()
    u3 = np.broadcast_to(U[:, :, None], (nz, ny, nx)).copy()
    T3 = np.broadcast_to(T[:, :, None], (nz, ny, nx)).copy()
    zero = np.zeros((nz, ny, nx))
    case.prim5 = np.ascontiguousarray(np.stack([d3, u3, zero, zero.copy(), T3]))
    case.di = np.ascontiguousarray(np.broadcast_to((Yk * rho[None])[:, :, :, None], (ns, nz, ny, nx)).copy())
    cmax = math.sqrt(1.4 * R0 / 0.029 * Tc)
    dmin = min(np.diff(x).min(), np.diff(y).min(), np.diff(z).min())
    case.dt = 0.5 * dmin / (Uj * (1 + pert) + cmax)
    case.nsteps = nsteps
    case.if_reaction = 1
    case.nsub = nsub
    case.info = dict(D=D, dmin=dmin)
    return case
