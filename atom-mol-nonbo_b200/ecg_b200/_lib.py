"""ctypes binding of libecgb200.so (declared in include/ecg_abi.h).

The shared library is built in this folder by build.py (nvcc, sm_100a).  If
it is missing, loading raises: there is no CPU fallback for the hot path.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libecgb200.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_vp = C.c_void_p

# name -> (restype, argtypes); the order mirrors include/ecg_abi.h
PROTOTYPES = {
    "ecg_ctx_create": (C.c_int, [C.c_int, _dp, _dp, C.c_int, _ip, _ip, C.c_int, C.c_int, C.c_char, C.c_int,
                                 C.POINTER(_vp)]),
    "ecg_ctx_destroy": (C.c_int, [_vp]),
    "ecg_set_params": (C.c_int, [_vp, _dp, C.c_int, C.c_int]),
    "ecg_set_params_device": (C.c_int, [_vp, C.c_void_p, C.c_int, C.c_int]),
    "ecg_compute_mat_elem": (C.c_int, [_vp, C.c_int, C.c_int, C.c_double]),
    "ecg_compute_mat_elem_and_deriv": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_double]),
    "ecg_ghepiis": (C.c_int, [_vp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, _dp, _dp, _ip]),
    "ecg_energy_ia": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, _dp,
                                _ip]),
    "ecg_energy_ib": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, _dp, _dp, _ip]),
    "ecg_energy_ib_adjoint": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, _dp,
                                        _dp, _ip]),
    "ecg_eval_candidates": (C.c_int, [_vp, C.c_int, C.c_int, _dp, C.c_double, C.c_double, C.c_int, _dp, _ip, _ip,
                                      _dp]),
    "ecg_eval_candidates_grad": (C.c_int, [_vp, C.c_int, C.c_int, _dp, C.c_double, C.c_double, C.c_int, _dp, _ip,
                                           _ip, _dp, _dp]),
    "ecg_energy_ga": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _dp, _ip]),
    "ecg_energy_gb": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp]),
    "ecg_energy_gb_adjoint": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp]),
    "ecg_overlap_penalty": (C.c_int, [_vp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, _dp, _dp]),
    "ecg_expectation_values": (C.c_int, [_vp, C.c_int, _dp, C.c_int, C.c_int, _ip, _ip, C.c_double, _dp, C.c_int,
                                         _dp, C.c_int, _dp, _dp, _dp, _dp, _dp]),
    "ecg_get_matrices": (C.c_int, [_vp, C.c_int, _dp, _dp, C.c_int, _dp, _dp, _dp]),
    "ecg_set_matrices": (C.c_int, [_vp, C.c_int, _dp, _dp, C.c_int, _dp, _dp]),
    "ecg_get_vectors": (C.c_int, [_vp, C.c_int, _dp, _dp]),
    "ecg_set_vectors": (C.c_int, [_vp, C.c_int, _dp, _dp]),
    "ecg_get_gradient": (C.c_int, [_vp, C.c_int, _dp]),
    "ecg_get_deriv": (C.c_int, [_vp, C.c_int, C.c_int, _dp]),
    "ecg_matrix_elements": (C.c_int, [_vp, C.c_int, _dp, _dp, _ip, C.c_int, _dp, _dp, _dp]),
    "ecg_launch_count": (C.c_longlong, [_vp]),
    "ecg_set_timing": (C.c_int, [_vp, C.c_int]),
    "ecg_get_stage_ms": (C.c_int, [_vp, _dp]),
    "ecg_sync": (C.c_int, [_vp]),
    "ecg_timer_start": (C.c_int, [_vp]),
    "ecg_timer_stop": (C.c_int, [_vp, _dp]),
    "ecg_pair_tiles": (C.c_int, [_vp, C.c_int, C.c_int, C.POINTER(C.c_longlong)]),
    "ecg_compute_mat_elem_tiles": (C.c_int, [_vp, C.c_int, C.c_int, C.c_double, C.c_longlong, C.c_longlong]),
    "ecg_pack_tiles": (C.c_int, [_vp, C.c_int, C.c_int, C.c_longlong, C.c_longlong, C.c_void_p]),
    "ecg_unpack_tiles": (C.c_int, [_vp, C.c_int, C.c_int, C.c_longlong, C.c_longlong, C.c_void_p]),
    "ecg_adjoint_part_doubles": (C.c_int, [_vp, C.POINTER(C.c_longlong)]),
    "ecg_adjoint_tiles": (C.c_int, [_vp, C.c_int, C.c_int, C.c_double, C.c_longlong, C.c_longlong, C.c_void_p]),
    "ecg_adjoint_finish": (C.c_int, [_vp, C.c_int, C.c_int, C.c_void_p, _dp]),
    "ecg_get_tuning": (C.c_int, [_vp, _ip, _ip, _ip, _dp]),
    "ecg_set_pivot_mode": (C.c_int, [_vp, C.c_int]),
    "ecg_set_wait_limit": (C.c_int, [_vp, C.c_int]),
    "ecg_set_factor_mode": (C.c_int, [_vp, C.c_int]),
    "ecg_factor_trace": (C.c_int, [_vp, C.c_int, C.c_void_p, C.c_longlong, C.POINTER(C.c_longlong)]),
    "ecg_ldl_schedule": (C.c_int, [C.c_int, C.c_int, C.c_void_p, C.c_longlong, C.POINTER(C.c_longlong)]),
    "ecg_io_bytes": (C.c_int, [_vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "ecg_probe_fp64_peak": (C.c_int, [C.c_int, _dp]),
    "ecg_probe_fp64_tensor_peak": (C.c_int, [C.c_int, _dp]),
    "ecg_adjoint_gradient_noalloc": (C.c_int, [C.c_int, _dp, _dp, C.c_int, _ip, _ip, C.c_void_p, C.c_void_p,
                                               C.c_void_p, C.c_double, C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
}

_lib = None


def load():
    """Load the library once; raises OSError if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing; build it with build.py (nvcc, sm_100a)")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def dptr(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def iptr(a):
    return a.ctypes.data_as(_ip) if a is not None else None
