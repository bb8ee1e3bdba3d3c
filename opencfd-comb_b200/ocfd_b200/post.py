"""Filtering and analysis parameters in the reference's layout, and the OCFD_analysis step.

Para%Filter(100,10) and Para%ANA_Para(100,10) (code/head/MODULE_parameter.f90:90-91) are stored
column-major, so group m is row m of a (10, 100) C-order array. The analysis type ids are the
reference's (MODULE_parameter.f90:28-29).
"""
import numpy as np

from . import files

FILTER_FO9P, FILTER_SHOCK = 1, 2
ANA_USER, ANA_TIME_AVERAGE, ANA_Q, ANA_BOX, ANA_SAVEDATA, ANA_CORNER = 99, 100, 101, 102, 103, 104

BOX_COLUMNS = ("tt", "Re_lamda", "Re_lamdax", "Amt", "vv_rms", "u_rms", "v_rms", "w_rms", "u_skewness",
               "u_flatness", "ux_skewness", "ux_flatness", "E_kinetic", "d_rms", "T_aver", "Amu_aver", "d_aver",
               "Ux_rms", "Alamdax")


def filter_table(groups):
    """(table, nfiltering) from a list of filter groups, each a dict with keys step (interval),
    x, y, z (1 = filter that direction), box = ((ib, ie), (jb, je), (kb, ke)) in global indices
    (default: everything), scheme (FILTER_FO9P / FILTER_SHOCK), s0 (amplitude, default 1) and
    rth (shock threshold, default 1e-5) -- the 13 entries of Filter(:, m) (OCFD_filtering.f90:23-43)."""
    if len(groups) > 10:
        raise ValueError("at most 10 filter groups (NFiltering <= 10)")
    t = np.zeros((10, 100))
    for m, g in enumerate(groups):
        box = g.get("box", ((1, 1 << 30), (1, 1 << 30), (1, 1 << 30)))
        t[m, 0] = g["step"]
        t[m, 1:4] = g.get("x", 0), g.get("y", 0), g.get("z", 0)
        t[m, 4:10] = box[0][0], box[0][1], box[1][0], box[1][1], box[2][0], box[2][1]
        t[m, 10] = g.get("scheme", FILTER_FO9P)
        t[m, 11] = g.get("s0", 1.0)
        t[m, 12] = g.get("rth", 1.0e-5)
    return t, len(groups)


def ana_table(entries):
    """(ANA_Para table, ANA_Number) from (kind, step interval, [ana_data ...]) entries."""
    if len(entries) > 10:
        raise ValueError("at most 10 analysis entries (ANA_Number <= 10)")
    t = np.zeros((10, 100))
    for m, e in enumerate(entries):
        kind, step = e[0], e[1]
        data = list(e[2]) if len(e) > 2 else []
        t[m, 0], t[m, 1] = kind, step
        t[m, 2:2 + len(data)] = data
    return t, len(entries)


def analysis(solver, istep, tt, table, n, outdir="."):
    """OCFD_analysis (code/others/OCFD_ANA.f90:3-33) after step istep: runs every due entry and
    writes what the reference writes (statistics.dat rows, Q-<Istep>.dat, the average files).
    Returns {kind: result} of what ran. ANA_SAVEDATA, ANA_Corner and user analyses are not built."""
    import os
    out = {}
    for m in range(n):
        kind, step = int(round(table[m, 0])), int(round(table[m, 1]))
        if step < 1 or istep % step != 0:
            continue
        data = table[m, 2:52]
        if kind == ANA_BOX:
            row = solver.ana_box(tt)
            with open(os.path.join(outdir, "statistics.dat"), "a") as fh:
                fh.write("".join("%20.12f" % x for x in row) + "\n")
            out[kind] = row
        elif kind == ANA_Q:
            q = solver.ana_q()
            files.write_3d_records(os.path.join(outdir, "Q-%07d.dat" % istep), [q])
            out[kind] = q
        elif kind == ANA_TIME_AVERAGE:
            k, t = solver.ana_time_average(solver.case.dt)
            if int(round(data[0])) > 0 and istep % int(round(data[0])) == 0:
                fields, k, t = solver.ana_average()
                files.write_average(os.path.join(outdir, "OCFD-comb%08d.dat.average" % istep), k, t, fields)
            out[kind] = (k, t)
        else:
            raise NotImplementedError("analysis kind %d is not built" % kind)
    return out
