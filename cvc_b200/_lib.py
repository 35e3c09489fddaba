"""ctypes binding of libcvcb200.so (the C ABI declared in include/cvcb.h).

The shared library is built in-tree (``make -C cvc_b200``); importing this
module without it raises immediately -- there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libcvcb200.so")

CVCB_OK = 0
CVCB_ERR_ARG = -1
CVCB_ERR_NULL = -2
CVCB_NO_CONVERGENCE = -3
CVCB_BREAKDOWN = -4
CVCB_ERR_STATE = -5
CVCB_ERR_NOMEM = -6
CVCB_ERR_CUDA = -7

PREC_DOUBLE, PREC_SINGLE, PREC_HALF = 0, 1, 2

_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_L = ctypes.c_long
_IP = ctypes.POINTER(ctypes.c_int)
_DP = ctypes.POINTER(ctypes.c_double)
_U32P = ctypes.POINTER(ctypes.c_uint32)


class SolverParams(ctypes.Structure):
    _fields_ = [
        ("precision", _I),
        ("link_recon", _I),
        ("block_rhs", _I),
        ("block_threads", _I),
        ("max_iter", _I),
        ("use_graph", _I),
        ("tol", _D),
        ("delta", _D),
    ]


class SolverStats(ctypes.Structure):
    _fields_ = [
        ("iterations", _I),
        ("reliable_updates", _I),
        ("restarts", _I),
        ("converged", _I),
        ("max_true_res", _D),
        ("seconds", _D),
        ("batch_rhs", _I),
    ]


# name -> (restype, argtypes); every symbol declared in include/cvcb.h
SIGNATURES = {
    "cvcb_last_error": (ctypes.c_char_p, []),
    "cvcb_version": (ctypes.c_char_p, []),
    "cvcb_geometry_tables": (_I, [_I, _I, _I, _I] + [_P] * 9),
    "cvcb_gamma_tables": (_I, [_P, _P]),
    "cvcb_boundary_phases": (_I, [_I, _I, _I, _I, _P, _P]),
    "cvcb_ranlxd": (_I, [_I, _I, _P, _L]),
    "cvcb_gauge_random": (_I, [_P, _I, _I, _I, _I, _D, _I]),
    "cvcb_lattice_create": (_I, [ctypes.POINTER(_P), _I, _I, _I, _I, _I]),
    "cvcb_lattice_destroy": (_I, [_P]),
    "cvcb_set_params": (_I, [_P, _D, _D, _P]),
    "cvcb_upload_gauge": (_I, [_P, _P]),
    "cvcb_gauge_unitarity": (_I, [_P, _DP]),
    "cvcb_Q_phi_tbc": (_I, [_P, _P, _P]),
    "cvcb_Hopping": (_I, [_P, _P, _P]),
    "cvcb_Qf5": (_I, [_P, _P, _P, _D]),
    "cvcb_Q_phi": (_I, [_P, _P, _P, _D]),
    "cvcb_g5_phi": (_I, [_P, _P]),
    "cvcb_mul_one_pm_imu_inv": (_I, [_P, _P, _D, _I]),
    "cvcb_spinor_scalar_product_co": (_I, [_P, _P, _P, _P, _I]),
    "cvcb_spinor_scalar_product_re": (_I, [_P, _P, _P, _P, _I]),
    "cvcb_spinor_scalar_product_co_noalloc": (_I, [_I, _P, _P, _P, _I, _P]),
    "cvcb_invert_Qtm": (_I, [_P, _P, _P, _D, _I, _P]),
    "cvcb_invert_Qtm_her": (_I, [_P, _P, _P, _D, _I, _P]),
    "cvcb_solver_defaults": (None, [ctypes.POINTER(SolverParams)]),
    "cvcb_solve": (_I, [_P, _P, _P, _I, ctypes.POINTER(SolverParams), ctypes.POINTER(SolverStats)]),
    "cvcb_time_stencil": (_I, [_P, _I, _I, _I, _I, _I, _DP]),
    "cvcb_sloppy_normal_op": (_I, [_P, _I, _I, _I, _I, _P, _P]),
    "cvcb_time_link_product": (_I, [_P, _I, _I, _DP, _DP]),
    "cvcb_tuned_shape": (_I, [_P, _I, _I, _I, _IP, _IP, _IP, _IP]),
    "cvcb_profile": (_I, [_P, _I]),
    "cvcb_counters": (_I, [_P, _P, _P, _P, _P]),
    "cvcb_cvc_contract": (_I, [_P, _P, _I, _P, _P]),
    "cvcb_cvc_ward": (_I, [_P, _P, _P]),
    "cvcb_p2gg_seq_source": (_I, [_P, _P, _P, _I, _P, _I, _I]),
    "cvcb_plaquette": (_I, [_P, _P, _P]),
    "cvcb_pi_momentum": (_I, [_P, _P, _I, _P, _P]),
    "cvcb_BHn": (_I, [_P, _P, _P, _I]),
    "cvcb_BH": (_I, [_P, _P, _P]),
    "cvcb_BH2": (_I, [_P, _P, _P]),
    "cvcb_BH3": (_I, [_P, _P, _P]),
    "cvcb_BH5": (_I, [_P, _P, _P]),
    "cvcb_BH7": (_I, [_P, _P, _P]),
    "cvcb_gamma5_BdagH4_gamma5": (_I, [_P, _P, _P, _P]),
    "cvcb_crc32": (_I, [ctypes.c_uint32, _P, ctypes.c_size_t, _U32P]),
    "cvcb_dml_checksum_accum": (_I, [_U32P, ctypes.c_uint64, _P, ctypes.c_size_t]),
    "cvcb_read_lime_gauge_field_doubleprec": (_I, [ctypes.c_char_p, _P, _I, _I, _I, _I, _U32P]),
    "cvcb_write_lime_gauge_field": (_I, [ctypes.c_char_p, _P, _I, _I, _I, _I, _I, _U32P]),
    "cvcb_read_lime_spinor": (_I, [_P, ctypes.c_char_p, _I, _I, _I, _I, _I, _U32P]),
    "cvcb_write_lime_spinor": (_I, [_P, ctypes.c_char_p, _I, _I, _I, _I, _I, _I, _U32P]),
    "cvcb_write_propagator": (_I, [_P, ctypes.c_char_p, _I, _I, _I, _I, _I, _U32P]),
    "cvcb_write_lime_contraction": (_I, [_P, ctypes.c_char_p, _I, _I, ctypes.c_char_p, _I, _I,
                                         _I, _I, _I, _I, _U32P]),
    "cvcb_read_lime_contraction": (_I, [_P, ctypes.c_char_p, _I, _I, _I, _I, _I, _I, _U32P]),
    "cvcb_pi_forward": (_I, [_P, _I, ctypes.POINTER(SolverParams), _D, _P, _P]),
    "cvcb_pi_tangent": (_I, [_P, _I, _P]),
    "cvcb_pi_backward": (_I, [_P, _P, _P, _P, _P]),
}

_lib = None


def load():
    """Load libcvcb200.so once; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            "libcvcb200.so is not built (run `make -C cvc_b200`); "
            "the package has no CPU fallback")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def ptr(x):
    """Address of a host numpy array, a torch tensor (host or CUDA) or an int."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if isinstance(x, np.ndarray):
        if not x.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be C-contiguous")
        return x.ctypes.data
    if hasattr(x, "data_ptr"):
        if not x.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return x.data_ptr()
    raise TypeError(f"cannot take the address of {type(x)!r}")


def ptr_array(fields):
    """A C array of pointers (double *const *) for a list of fields."""
    arr = (ctypes.c_void_p * len(fields))()
    for i, f in enumerate(fields):
        arr[i] = ptr(f)
    return arr


def last_error():
    return load().cvcb_last_error().decode(errors="replace")
