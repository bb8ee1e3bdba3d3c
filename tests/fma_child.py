"""Child process of test_gpu_fma.py: runs the protocol cases through the library variant that
OCFD_B200_LIB selects and writes each case's final state and per-step hybrid sensor to an npz.

  OCFD_B200_LIB=fma python tests/fma_child.py <out_dir> <case> [<case> ...]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "opencfd-comb_b200"))

from ocfd_b200 import abi, cases, solver  # noqa: E402


def protocol_cases():
    """name -> (case builder, steps, if_reaction, nsub)"""
    return {
        "isotropic16_weno5": (lambda: cases.isotropic(n=16), 10, 0, 1),
        "flatplate_hybrid": (lambda: cases.flatplate(nx=40, ny=24, nz=12, scheme="HYBRID", lx=0.01, ly=0.004,
                                                     y1=2e-5), 10, 0, 1),
        "flatplate_omp6": (lambda: cases.flatplate(nx=40, ny=24, nz=12, scheme="OMP6", lx=0.01, ly=0.004,
                                                   y1=2e-5), 10, 0, 1),
        "jet24": (lambda: cases.jet(nx=24, ny=16, nz=16), 10, 1, 1),
    }


def main():
    out = sys.argv[1]
    for name in sys.argv[2:]:
        builder, steps, ifr, nsub = protocol_cases()[name]
        c = builder()
        g = solver.Solver(c)
        g.init_state()
        rh = []
        for s in range(steps):
            g.tt = s * c.dt
            g.step(c.dt, ifr, nsub)
            if c.params.scheme_invis == abi.SCHEME_HYBRID:
                rh.append(g.rhybrid())
        f, di, pr = g.download_state()
        g.close()
        np.savez(os.path.join(out, name + ".npz"), f=f, di=di, prims=pr,
                 rh=np.array(rh) if rh else np.zeros(0), variant=solver.VARIANT)
    print("done", solver.VARIANT)


if __name__ == "__main__":
    main()
