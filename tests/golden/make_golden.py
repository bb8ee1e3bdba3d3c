"""Writes the golden fixtures of tests/golden/ with the CPU oracle.

The reference's own tests hold no output vectors (its CTest cases check exit codes only) and the
Fortran cannot be compiled here, so these fixtures record the oracle's results on small seeded
cases. tests/test_golden.py checks that the oracle still reproduces them bit for bit (guarding
the restatement against regressions) and the GPU tests compare the CUDA path with the same files.

Run: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "opencfd-comb_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import pyoracle  # noqa: E402
from ocfd_b200 import cases  # noqa: E402

L = 4


def golden_cases():
    """name -> (case builder, steps, if_reaction, nsub)"""
    names, *_ = cases.h2air_structs()
    Y = [1e-6, 0.2, 0.02, 0.1, 1e-5, 1e-6, 1e-7, 1e-7, 0.68]
    return {
        "isotropic12_weno5": (lambda: cases.isotropic(n=12), 2, 0, 1),
        "isotropic12_omp6": (lambda: cases.isotropic(n=12, scheme="OMP6"), 2, 0, 1),
        "flatplate_hybrid": (lambda: cases.flatplate(nx=32, ny=16, nz=8, scheme="HYBRID", lx=0.01, ly=0.004,
                                                     y1=2e-5), 2, 0, 1),
        "isotropic10_o2n2": (lambda: cases.isotropic(n=10, species=["O2", "N2"], Y=[0.233, 0.767]), 2, 0, 1),
        "isotropic8_h2air": (lambda: cases.isotropic(n=8, species=names, Y=Y, wilke=True, T0=1500.0), 1, 1, 2),
    }


def run(builder, steps, if_reaction, nsub):
    c = builder()
    o = pyoracle.OracleSolver(c)
    o.init_state()
    for s in range(steps):
        o.step(c.dt, s * c.dt, if_reaction, nsub)
    f, di, pr = o.download_state()
    o.close()
    return c, f, di[:, L:-L, L:-L, L:-L].copy(), pr[:, L:-L, L:-L, L:-L].copy()


def main():
    for name, (builder, steps, ifr, nsub) in golden_cases().items():
        c, f, di, pr = run(builder, steps, ifr, nsub)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, f=f, di=di, prims=pr, dt=c.dt, steps=steps, if_reaction=ifr, nsub=nsub)
        print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
