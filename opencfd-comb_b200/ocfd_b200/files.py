"""Readers and writers for the reference's case-file formats.

The Fortran driver keeps reading these itself; this host mirror reads them so that the
synthetic workloads, the tests and the bench can build the ABI structs from the same files.

  specie.in                     read_Spec   code/Chemical/CHEM_thermdyn.f90:16-51
  Reaction.in                   read_Reac   code/Chemical/CHEM_reactions.f90:15-69
  viscosity.in / conductivity.in / diffusion_coefficients.in
                                read_*_coefficients code/Chemical/TRANSPORT_modules.f90:82-251
  opencfd-comb2.in (&control_opencfd namelist subset)
                                read_control_parameter code/mpi-io/OCFD_readpara.f90:26-110
  Fortran unformatted sequential records (grid, restart)
                                read_3d / write_3d code/mpi-io/OCFD_IO_mpi.f90:151-307
"""
import re
import struct

import numpy as np

_num = re.compile(r"[dD]")


def _tokens(line):
    """List-directed tokens of one record (commas or blanks separate, 'd' exponents)."""
    line = line.split("!")[0]
    out = []
    for t in re.split(r"[,\s]+", line.strip()):
        if t:
            out.append(t)
    return out


def _f(t):
    return float(_num.sub("e", t))


def _strip_q(t):
    return t.strip().strip("'\"").strip()


def read_specie(path):
    """Returns dict(n_tct, tct[], tct_max, species=[dict(name, mi, spec_flag, coef[n_tct][7])])."""
    lines = open(path, encoding="latin-1").read().splitlines()
    # header: 2 comment records, then N_Tct, Tct(1..N_Tct-1), Tct_max, then 1 comment record
    it = iter(lines)
    next(it), next(it)
    t = _tokens(next(it))
    n_tct = int(t[0])
    tct = [_f(x) for x in t[1:n_tct]]
    tct_max = _f(t[n_tct])
    next(it)
    species = []
    rest = [ln for ln in it]
    pos = 0

    def nonblank():
        nonlocal pos
        while pos < len(rest) and not rest[pos].strip():
            pos += 1
        if pos >= len(rest):
            return None
        ln = rest[pos]
        pos += 1
        return ln

    while True:
        # one comment record before each species
        ln = nonblank()
        if ln is None:
            break
        if ln.strip().startswith("#"):
            ln = nonblank()
            if ln is None or ln.strip().startswith("#"):
                break
        name = _strip_q(ln)
        t = _tokens(nonblank())
        mi = _f(t[0])
        flag = int(_f(t[1])) if len(t) > 1 and "." not in t[1] else (1 if name in ("O", "H", "N", "AR", "HE") else 2)
        coef = []
        for _ in range(n_tct):
            vals = []
            while len(vals) < 7:
                vals += [_f(x) for x in _tokens(nonblank())]
            coef.append(vals[:7])
        species.append(dict(name=name, mi=mi, spec_flag=flag, coef=coef))
    return dict(n_tct=n_tct, tct=tct, tct_max=tct_max, species=species)


def read_reaction(path):
    """Reaction.in. Files written before the reverse-rate record was added (ReReac=0 with no
    placeholder line, as in cases/jet/Reaction.in) are accepted: a stoichiometric row is
    recognised by holding exactly N_spec integers."""
    lines = [ln for ln in open(path, encoding="latin-1").read().splitlines()]
    pos = 2
    t = _tokens(lines[pos]); pos += 1
    ns, nr, rereac = int(t[0]), int(t[1]), int(t[2])
    names = _tokens(lines[pos + 1])
    pos += 4
    reacs = []

    def is_int_row(ln):
        tt = _tokens(ln)
        return len(tt) == ns and all(re.fullmatch(r"-?\d+", x) for x in tt)

    for j in range(nr):
        pos += 1  # comment
        eqn = lines[pos].strip(); pos += 1
        t = _tokens(lines[pos]); pos += 1
        r = dict(eqn=eqn, af_type=int(t[0]), tr_reac=int(t[1]), fc_troe=_f(t[2]))
        a = [_f(x) for x in _tokens(lines[pos])]; pos += 1
        r["arr"] = [a[:3]]
        if r["af_type"] != 0:
            a = [_f(x) for x in _tokens(lines[pos])]; pos += 1
            r["arr"].append(a[:3])
        else:
            r["arr"].append([0.0, 0.0, 0.0])
        r["rev"] = [0.0, 0.0, 0.0]
        r["park"] = [0.0] * 5
        if rereac == 0:
            if not is_int_row(lines[pos]):
                pos += 1
        elif rereac == 1:
            r["rev"] = [_f(x) for x in _tokens(lines[pos])][:3]; pos += 1
        else:
            r["park"] = [_f(x) for x in _tokens(lines[pos])][:5]; pos += 1
        r["vf"] = [int(x) for x in _tokens(lines[pos])]; pos += 1
        r["vr"] = [int(x) for x in _tokens(lines[pos])]; pos += 1
        if r["tr_reac"] == 1:
            r["treff"] = [_f(x) for x in _tokens(lines[pos])]; pos += 1
        else:
            r["treff"] = [0.0] * ns
        reacs.append(r)
    return dict(n_spec=ns, n_reac=nr, rereac=rereac, species=names, reactions=reacs)


def read_fit_by_name(path, ncoef=4):
    """viscosity.in / conductivity.in: 2 comments, N, then (name, coefficients) records."""
    lines = [ln for ln in open(path, encoding="latin-1").read().splitlines() if ln.strip()]
    n = int(_tokens(lines[2])[0])
    out = {}
    pos = 3
    for _ in range(n):
        name = _strip_q(lines[pos]); pos += 1
        out[name] = [_f(x) for x in _tokens(lines[pos])][:ncoef]; pos += 1
    return out


def read_diffusion(path):
    lines = [ln for ln in open(path, encoding="latin-1").read().splitlines() if ln.strip()]
    n = int(_tokens(lines[4])[0])
    out = {}
    pos = 5
    for _ in range(n):
        a, b = [_strip_q(x) for x in lines[pos].split()[:2]]; pos += 1
        out[(a, b)] = [_f(x) for x in _tokens(lines[pos])][:4]; pos += 1
    return out


def read_namelist(path, group="control_opencfd"):
    """Minimal &group ... /$end reader for the scalar and array keys of opencfd-comb2.in."""
    txt = open(path, encoding="latin-1").read()
    m = re.search(r"[&$]" + group + r"(.*?)(?:\$end|/\s*$|&end)", txt, re.S | re.I)
    body = m.group(1)
    body = "\n".join(ln.split("!")[0] for ln in body.splitlines())
    out = {}
    for key, val in re.findall(r"([A-Za-z_][A-Za-z0-9_]*(?:\(\s*:\s*,\s*\d+\s*\))?)\s*=\s*(.*?)(?=\s+[A-Za-z_][A-Za-z0-9_]*(?:\(\s*:\s*,\s*\d+\s*\))?\s*=|\Z)", body, re.S):
        vals = []
        for t in _tokens(val):
            t = t.strip()
            if t.startswith(("'", '"')):
                vals.append(_strip_q(t))
            else:
                try:
                    vals.append(int(t) if re.fullmatch(r"-?\d+", t) else _f(t))
                except ValueError:
                    vals.append(t)
        out[key.strip().lower()] = vals[0] if len(vals) == 1 else vals
    return out


# ---------------- Fortran unformatted sequential records ----------------

def write_records(path, arrays):
    """Each array becomes one record: 4-byte length, payload, 4-byte length (gfortran default)."""
    with open(path, "wb") as fh:
        for a in arrays:
            b = np.ascontiguousarray(a).tobytes()
            fh.write(struct.pack("<i", len(b)))
            fh.write(b)
            fh.write(struct.pack("<i", len(b)))


def read_records(path, dtype=np.float64):
    out = []
    with open(path, "rb") as fh:
        while True:
            h = fh.read(4)
            if len(h) < 4:
                break
            n = struct.unpack("<i", h)[0]
            out.append(fh.read(n))
            if struct.unpack("<i", fh.read(4))[0] != n:
                raise ValueError("corrupt Fortran record marker in %s" % path)
    return out


def write_restart(path, istep, tt, fields):
    """save_flow_data layout (OCFD_IO.f90:39-64): header (int32 Istep, real64 tt), then every
    field as nz records of nx*ny doubles. fields: list of (nx,ny,nz) Fortran-ordered arrays."""
    with open(path, "wb") as fh:
        hdr = struct.pack("<id", istep, tt)
        fh.write(struct.pack("<i", len(hdr))); fh.write(hdr); fh.write(struct.pack("<i", len(hdr)))
        for f in fields:
            f = np.asarray(f, dtype=np.float64)
            for k in range(f.shape[2]):
                b = np.asfortranarray(f[:, :, k]).tobytes(order="F")
                fh.write(struct.pack("<i", len(b))); fh.write(b); fh.write(struct.pack("<i", len(b)))


def read_restart(path, nx, ny, nz, nfields):
    recs = read_records(path)
    istep, tt = struct.unpack("<id", recs[0])
    fields = []
    for m in range(nfields):
        arr = np.empty((nx, ny, nz), order="F")
        for k in range(nz):
            arr[:, :, k] = np.frombuffer(recs[1 + m * nz + k], dtype=np.float64).reshape((nx, ny), order="F")
        fields.append(arr)
    return istep, tt, fields


def _write_planes(fh, a):
    """write_3d (OCFD_IO_mpi.f90:232): one record of nx*ny doubles per k plane; a is (nz, ny, nx)
    in C order, whose planes are the Fortran (nx, ny) column-major planes."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    n = struct.pack("<i", a[0].nbytes)
    for k in range(a.shape[0]):
        fh.write(n); fh.write(memoryview(a[k]).cast("B")); fh.write(n)  # no copy of the plane


def write_3d_records(path, arrays):
    """Files written by write_3d alone, e.g. Q-<Istep>.dat of ana_getQ (OCFD_ANA.f90:183-188)."""
    with open(path, "wb") as fh:
        for a in arrays:
            _write_planes(fh, a)


def write_average(path, k_average, t_average, fields):
    """OCFD-comb<Istep>.dat.average of ana_time_average (OCFD_ANA.f90:119-139): header record
    (int32 K_average, real64 t_average), then dm, um, vm, wm, Tm and every diav as write_3d."""
    with open(path, "wb") as fh:
        hdr = struct.pack("<id", k_average, t_average)
        fh.write(struct.pack("<i", len(hdr))); fh.write(hdr); fh.write(struct.pack("<i", len(hdr)))
        for a in fields:
            _write_planes(fh, a)


def read_average(path, nx, ny, nz, nfields):
    recs = read_records(path)
    k_average, t_average = struct.unpack("<id", recs[0])
    out = np.empty((nfields, nz, ny, nx))
    for m in range(nfields):
        for k in range(nz):
            out[m, k] = np.frombuffer(recs[1 + m * nz + k], dtype=np.float64).reshape(ny, nx)
    return k_average, t_average, out


def write_flow_data(path, istep, tt, fields):
    """save_flow_data (OCFD_IO.f90:39-64): header record (int32 Istep, real64 tt), then d, u, v, w,
    T and every di as write_3d1 planes; fields is (5 + Ns, nz, ny, nx) in C order."""
    with open(path, "wb") as fh:
        hdr = struct.pack("<id", istep, tt)
        fh.write(struct.pack("<i", len(hdr))); fh.write(hdr); fh.write(struct.pack("<i", len(hdr)))
        for a in fields:
            _write_planes(fh, a)


def read_flow_data(path, nx, ny, nz, ns):
    """read_flow_data (OCFD_IO.f90:5-36): (Istep, tt, (5 + ns, nz, ny, nx) array)."""
    k, t, a = read_average(path, nx, ny, nz, 5 + ns)
    return k, t, a
