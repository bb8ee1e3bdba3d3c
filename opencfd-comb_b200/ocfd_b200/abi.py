"""ctypes mirror of include/ocfd_gpu.h (the C ABI of the B200 hot path).

The structs carry what the reference's Fortran driver holds in its Para / Scheme / SPEC /
REAC / Trans records (code/head/MODULE_parameter.f90:49-96, code/Chemical/CHEM_modules.f90:34-67,
code/Chemical/TRANSPORT_modules.f90:16-22) after read_parameter (code/mpi-io/OCFD_readpara.f90:5-20).
"""
import ctypes as C

MAX_SPEC = 16
MAX_REAC = 64
NTCT_MAX = 10

OK = 0
ERR_PARAM = -1
ERR_CUDA = -2
ERR_NAN = -3
ERR_NEGATIVE_ET = -4
ERR_STATE = -5
ERR_TIMEOUT = -6
ERR_UNSUPPORTED = -7
ERR_CHEM = -8

SCHEME_WENO5, SCHEME_WENO7, SCHEME_OMP6, SCHEME_UD7L = 1, 2, 3, 4
SCHEME_CD6, SCHEME_CD8, SCHEME_HYBRID = 5, 6, 10
SPLIT_SW, SPLIT_LLF = 1, 2
BC_NONE, BC_BOUNDARYLAYER, BC_JET = 0, 2, 4
CHEM_EULER, CHEM_RK2, CHEM_RK3, CHEM_IMPLICIT = 1, 2, 3, -1

SCHEME_NAMES = {"WENO5": SCHEME_WENO5, "WENO7": SCHEME_WENO7, "OMP6": SCHEME_OMP6, "UD7L": SCHEME_UD7L,
                "CD6": SCHEME_CD6, "CD8": SCHEME_CD8, "HYBRID": SCHEME_HYBRID}
BC_NAMES = {"BC_NONE": BC_NONE, "BC_BOUNDARYLAYER": BC_BOUNDARYLAYER, "BC_JET": BC_JET}

D = C.c_double
I = C.c_int


class Params(C.Structure):
    _fields_ = [
        ("nx", I), ("ny", I), ("nz", I), ("lap", I), ("n_spec", I),
        ("iperiodic", I * 3),
        ("periodic_span", (D * 3) * 3),
        ("scheme_invis", I), ("scheme_vis", I),
        ("scheme_boundary", I * 6),
        ("ghost_cell", I * 6),
        ("if_scheme_character", I), ("if_viscous", I), ("flux_splitting", I), ("if_mass_force", I),
        ("mass_force", D * 3),
        ("ibc", I),
        ("bc_para", D * 100),
        ("hybrid_para", D * 100),
        ("ud7l_diss", D), ("aoa", D),
        ("if_realgas", I), ("chem_timeadv", I), ("wall_catalysis", I), ("istep_show", I),
    ]


class Thermo(C.Structure):
    _fields_ = [
        ("n_spec", I), ("n_tct", I),
        ("tct", D * NTCT_MAX), ("tct_max", D),
        ("mi", D * MAX_SPEC), ("spec_flag", I * MAX_SPEC),
        ("coef", ((D * 7) * NTCT_MAX) * MAX_SPEC),
    ]


class Kinetics(C.Structure):
    _fields_ = [
        ("n_spec", I), ("n_reac", I), ("rereac", I),
        ("af_type", I * MAX_REAC), ("tr_reac", I * MAX_REAC), ("fc_troe", D * MAX_REAC),
        ("af", (D * 2) * MAX_REAC), ("bf", (D * 2) * MAX_REAC), ("ef", (D * 2) * MAX_REAC),
        ("ar", D * MAX_REAC), ("br", D * MAX_REAC), ("er", D * MAX_REAC),
        ("park", (D * 5) * MAX_REAC),
        ("vf", (I * MAX_SPEC) * MAX_REAC), ("vr", (I * MAX_SPEC) * MAX_REAC),
        ("treff", (D * MAX_SPEC) * MAX_REAC),
    ]


class Transport(C.Structure):
    _fields_ = [
        ("flag_vis", I), ("flag_cond", I), ("flag_diff", I),
        ("amu0", D), ("pr", D), ("sc", D), ("amk0", D),
        ("mu_an", (D * 5) * MAX_SPEC),
        ("k_an", (D * 5) * MAX_SPEC),
        ("d_an", ((D * 4) * MAX_SPEC) * MAX_SPEC),
    ]


class BcData(C.Structure):
    _fields_ = [
        ("inlet", C.POINTER(D)), ("upper", C.POINTER(D)), ("wall_pertb", C.POINTER(D)),
        ("n_tm", I), ("tm", C.POINTER(D)), ("fait", C.POINTER(D)),
    ]


def dptr(a):
    """double* of a C-contiguous float64 numpy array (None -> NULL)."""
    if a is None:
        return None
    assert a.dtype.name == "float64" and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(D))


def iptr(a):
    if a is None:
        return None
    assert a.dtype.name == "int32" and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(I))


# exported symbols of libocfd_gpu.so with their ctypes signatures
PD = C.POINTER(D)
PI = C.POINTER(I)
GPU_SIGNATURES = {
    "ocfd_gpu_init": (I, [C.POINTER(Params), C.POINTER(Thermo), C.POINTER(Kinetics), C.POINTER(Transport),
                          C.POINTER(BcData), PD, PD]),
    "ocfd_gpu_upload_state": (I, [PD, PD, PD]),
    "ocfd_gpu_flow_advance": (I, [D, D]),
    "ocfd_gpu_chem_advance": (I, [D, I]),
    "ocfd_gpu_step": (I, [D, D, I, I]),
    "ocfd_gpu_download_state": (I, [PD, PD, PD]),
    "ocfd_gpu_diag": (I, [PD, PD]),
    "ocfd_gpu_download_rhybrid": (I, [PD]),
    "ocfd_gpu_download_metrics": (I, [PD]),
    "ocfd_gpu_chem_batch": (I, [I, PD, PD, PD, PI]),
    "ocfd_gpu_chem_batch_device": (I, [I, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ocfd_gpu_stats": (I, [C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "ocfd_gpu_last_error": (C.c_char_p, []),
    "ocfd_gpu_finalize": (I, []),
    "ocfd_gpu_fp64_peak_gflops": (D, []),
    "ocfd_gpu_init_state": (I, [PD, PD, D]),
    "ocfd_gpu_run": (I, [D, D, I, I, I]),
    "ocfd_gpu_chem_setup": (I, [C.POINTER(Thermo), C.POINTER(Kinetics), I, I]),
    "ocfd_gpu_diag_begin": (I, []),
    "ocfd_gpu_diag_end": (I, [PD, PD]),
    "ocfd_gpu_snapshot": (I, [I, D]),
    "ocfd_gpu_snapshot_wait": (I, [PI, PD, C.POINTER(PD)]),
    "ocfd_gpu_surrogate_fused": (I, [I]),
    "ocfd_gpu_filtering": (I, [I, I, PD, PI]),
    "ocfd_gpu_keep_viscosity": (I, [I]),
    "ocfd_gpu_ana_box": (I, [D, PD]),
    "ocfd_gpu_ana_q": (I, [PD]),
    "ocfd_gpu_ana_time_average": (I, [D, PI, PD]),
    "ocfd_gpu_ana_average": (I, [I, PD, PI, PD]),
    "ocfd_gpu_autotune": (I, [I, PI, PD]),
    "ocfd_gpu_set_tiles": (I, [PI]),
    "ocfd_gpu_get_tiles": (I, [PI]),
    "ocfd_gpu_profile": (I, [I]),
    "ocfd_gpu_profile_read": (I, [I, PD, C.POINTER(C.c_longlong)]),
    "ocfd_gpu_profile_name": (C.c_char_p, [I]),
    "ocfd_gpu_profile_nclass": (I, []),
    "ocfd_gpu_stream": (C.c_void_p, []),
    "ocfd_gpu_launch_count": (C.c_longlong, []),
    "ocfd_gpu_is_separable": (I, []),
    "ocfd_gpu_device_bytes": (C.c_longlong, []),
    "ocfd_gpu_event_record": (I, [I]),
    "ocfd_gpu_event_elapsed": (I, [I, I, PD]),
    "ocfd_gpu_pinned_alloc": (I, [C.c_size_t, C.POINTER(C.c_void_p)]),
    "ocfd_gpu_pinned_free": (I, [C.c_void_p]),
    "ocfd_gpu_step_launches": (I, []),
    "ocfd_gpu_chem_batch_noalloc": (I, [I, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ocfd_gpu_chem_batch_status": (I, [C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "ocfd_gpu_chem_constant_pressure": (I, [I]),
    "ocfd_gpu_chem_compiled_mechanism": (I, [I]),
    "ocfd_gpu_gemm_bf16": (I, [I, I, I, C.c_void_p, C.c_longlong, C.c_longlong, C.c_void_p, C.c_longlong,
                               C.c_longlong, C.c_void_p, C.c_longlong, C.c_void_p, I, I]),
    "ocfd_gpu_surrogate_init": (I, [C.c_uint]),
    "ocfd_gpu_surrogate_train": (I, [I, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, PD, I, I, D,
                                     C.c_uint, PD]),
    "ocfd_gpu_surrogate_predict": (I, [I, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p]),
    "ocfd_gpu_chem_batch_surrogate": (I, [I, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, D, PI]),
    "ocfd_gpu_surrogate_blob": (C.c_longlong, [C.POINTER(C.c_float), C.c_longlong, I]),
    "ocfd_gpu_surrogate_grad": (I, [I, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float), PD]),
    "ocfd_gpu_chem_temperature": (I, [I, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ocfd_gpu_chem_mode": (I, [I, D]),
    "ocfd_gpu_chem_surrogate_rejected": (C.c_longlong, [C.POINTER(C.c_longlong)]),
}
