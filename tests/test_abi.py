"""The C ABI library (libocfd_gpu.so) loads without a GPU and exports every entry point that
include/ocfd_gpu.h declares; the ctypes mirror matches the header's struct layouts."""
import ctypes as C
import os
import re

import pytest

from ocfd_b200 import abi
from ocfd_b200 import solver

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ocfd_gpu.h")


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(ocfd_gpu_\w+)\s*\(", txt)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("ocfd_gpu_init", "ocfd_gpu_upload_state", "ocfd_gpu_flow_advance", "ocfd_gpu_chem_advance",
                 "ocfd_gpu_download_state", "ocfd_gpu_diag", "ocfd_gpu_last_error", "ocfd_gpu_finalize"):
        assert must in names


def test_library_exports_every_declared_symbol():
    if not os.path.exists(solver.LIBPATH):
        pytest.skip("libocfd_gpu.so not built")
    lib = C.CDLL(solver.LIBPATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_ctypes_struct_sizes_match_c():
    """Compile a tiny C program against the header and compare sizeof / offsetof."""
    import subprocess
    import tempfile
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "ocfd_gpu.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu\n", sizeof(ocfd_params), sizeof(ocfd_thermo), sizeof(ocfd_kinetics),
         sizeof(ocfd_transport), sizeof(ocfd_bcdata));
  printf("%zu %zu %zu\n", offsetof(ocfd_params, bc_para), offsetof(ocfd_params, hybrid_para),
         offsetof(ocfd_params, istep_show));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        cfile = os.path.join(d, "s.c")
        open(cfile, "w").write(src)
        exe = os.path.join(d, "s")
        subprocess.check_call(["gcc", "-I", os.path.dirname(HEADER), cfile, "-o", exe])
        out = subprocess.check_output([exe]).decode().split()
    sizes = [int(x) for x in out]
    assert sizes[:5] == [C.sizeof(abi.Params), C.sizeof(abi.Thermo), C.sizeof(abi.Kinetics),
                         C.sizeof(abi.Transport), C.sizeof(abi.BcData)]
    assert sizes[5:] == [abi.Params.bc_para.offset, abi.Params.hybrid_para.offset, abi.Params.istep_show.offset]


def test_product_fails_loudly_without_device():
    """No CPU fallback: without a CUDA device the library refuses to initialise."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    if not os.path.exists(solver.LIBPATH):
        pytest.skip("libocfd_gpu.so not built")
    from ocfd_b200 import cases
    c = cases.isotropic(n=8)
    with pytest.raises(solver.OcfdError) as ei:
        solver.Solver(c)
    assert ei.value.code == abi.ERR_CUDA
