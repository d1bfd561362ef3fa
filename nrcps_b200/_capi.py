"""ctypes bindings of libnrcps_b200.so (the C ABI declared in include/nrcps_b200.h).

The shared library is built in-tree by ``python -m nrcps_b200.build``.  There
is no fallback: if the library is missing or a CUDA call fails, the calls
below raise.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnrcps_b200.so")

OK = 0
STATUS_NAMES = {0: "OK", 1: "INVALID_ARGUMENT", 2: "UNSUPPORTED", 3: "CUDA", 4: "OUT_OF_MEMORY",
                5: "SINGULAR", 6: "NONFINITE", 7: "TIMEOUT"}
F64, F32 = 0, 1
RNG_KINDS = {"RAN0": 0, "RAN1": 1, "RAN2": 2, "RAN3": 3, "RANLXS0": 4, "RANLXS1": 5, "RANLXS2": 6,
             "RANLXD1": 7, "RANLXD2": 8}
FIELD_KINDS = {"GAUSS": 0, "COMPLEXGAUSS": 1, "ZTWO": 2, "ZTHREE": 3}
DISP_TYPES = {"STANDARD": 0, "QUADRATIC": 1, "PERFECT": 2}
INTERACTION_TYPES = {"NONE": 0, "XISQMINUSONE": 1, "ONEMINUSXIINVSQ": 2}
POTENTIAL_TYPES = {"LIN": 0, "EXP": 1}
WAVEFUNC_TYPES = {"NONE": 0, "UNIFORM": 1, "GND": 2, "TGND": 3, "PAIR1": 4, "PAIR2": 5}


class NrcpsError(RuntimeError):
    """A non-OK nrcps_status, with the library's description."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class PositionFactor(ctypes.Structure):
    _fields_ = [("field_mode", ctypes.c_int), ("dev_field", ctypes.c_void_p), ("bit0", ctypes.c_uint64),
                ("conf_stride", ctypes.c_uint64), ("a", ctypes.c_double), ("dev_pos", ctypes.c_void_p),
                ("dev_conf_base", ctypes.c_void_p)]


class Job(ctypes.Structure):
    _fields_ = [("dims", ctypes.c_int * 3), ("T", ctypes.c_int), ("n_orb", ctypes.c_int), ("n_conf", ctypes.c_int),
                ("rng_kind", ctypes.c_int), ("seed", ctypes.c_long), ("field_kind", ctypes.c_int),
                ("mode", ctypes.c_int), ("precision", ctypes.c_int), ("plane_wave", ctypes.c_int),
                ("use_potential", ctypes.c_int), ("qr_period", ctypes.c_int), ("a", ctypes.c_double),
                ("local_interaction", ctypes.c_int)]


class BatchJob(ctypes.Structure):
    _fields_ = [("L", ctypes.c_int), ("n_orb", ctypes.c_int), ("T", ctypes.c_int), ("n_conf", ctypes.c_int),
                ("pw_index", ctypes.POINTER(ctypes.c_int)), ("kin_xi", ctypes.POINTER(ctypes.c_double))]


class BranchParams(ctypes.Structure):
    _fields_ = [("dims", ctypes.c_int * 3), ("levels", ctypes.c_int), ("branches", ctypes.c_int),
                ("steps", ctypes.c_int), ("rng_kind", ctypes.c_int), ("seed", ctypes.c_long),
                ("field_kind", ctypes.c_int), ("precision", ctypes.c_int), ("a", ctypes.c_double)]


class BatchParams(ctypes.Structure):
    _fields_ = [("rng_kind", ctypes.c_int), ("seed", ctypes.c_long), ("field_kind", ctypes.c_int),
                ("precision", ctypes.c_int), ("a", ctypes.c_double), ("qr_period", ctypes.c_int)]


# Every exported symbol with its argument and result types.
_P = ctypes.c_void_p
_I = ctypes.c_int
_L = ctypes.c_long
_D = ctypes.c_double
_U64 = ctypes.c_uint64
_IP = ctypes.POINTER(ctypes.c_int)
_DP = ctypes.POINTER(ctypes.c_double)
_LP = ctypes.POINTER(ctypes.c_long)
SIGNATURES = {
    "nrcps_create": ([_I, ctypes.POINTER(_P)], _I),
    "nrcps_destroy": ([_P], _I),
    "nrcps_last_error": ([_P], ctypes.c_char_p),
    "nrcps_set_stream": ([_P, _P], _I),
    "nrcps_synchronize": ([_P], _I),
    "nrcps_version": ([], ctypes.c_char_p),
    "nrcps_set_option": ([_P, ctypes.c_char_p, _L], _I),
    "nrcps_autotune": ([_P, _I, _I, _IP], _I),
    "nrcps_fused_choice": ([_P, _I, _I, _IP, _IP], _I),
    "nrcps_dispersion_table": ([_IP, _I, _D, _I, _D, _DP], _I),
    "nrcps_kinetic_table": ([_IP, _I, _D, _D, _D, _DP], _I),
    "nrcps_interaction_table": ([_IP, _D, _I, _DP, _I, _D, _D, _DP], _I),
    "nrcps_potential_table": ([_IP, _I, _D, _D, _D, _D, _DP], _I),
    "nrcps_momenta": ([_IP, _I, _D, _D, _D, _I, _IP, _DP, _IP, _IP], _I),
    "nrcps_sho_source": ([_IP, _D, _D, _D, _DP, _DP], _I),
    "nrcps_two_body_tables": ([_IP, _I, _I, _I, _D, _D, _D, _D, _DP, _IP], _I),
    "nrcps_rng_seed_state": ([_I, _L, _LP, _IP], _I),
    "nrcps_rng_skip": ([_I, _LP, _U64], _I),
    "nrcps_rng_uniforms": ([_P, _I, _L, _U64, _U64, _P], _I),
    "nrcps_draw_fields": ([_P, _I, _L, _I, _L, _L, ctypes.POINTER(_U64), _P], _I),
    "nrcps_draw_z2_bits": ([_P, _I, _L, _U64, _U64, _P], _I),
    "nrcps_fft3d": ([_P, _P, _I, _IP, _I, _I], _I),
    "nrcps_kinetic_evolve": ([_P, _P, _I, _L, _P, _I], _I),
    "nrcps_potential_evolve": ([_P, _P, _I, _IP, _P, _I], _I),
    "nrcps_interaction_initialize": ([_P, _P, _P, _IP, _P], _I),
    "nrcps_interaction_evolve": ([_P, _P, _I, _IP, _P, _I], _I),
    "nrcps_propagate": ([_P, _P, _I, _I, _IP, _P, ctypes.POINTER(PositionFactor), _I], _I),
    "nrcps_overlap": ([_P, _P, _I, _P, _I, _I, _L, _I, _P], _I),
    "nrcps_overlap_planewave": ([_P, _P, _I, _P, _I, _I, _L, _I, _P], _I),
    "nrcps_pair_matrix": ([_P, _P, _P, _I, _I, _L, _P, _P, _I, _P], _I),
    "nrcps_inner_product_ptrs": ([_P, _P, _P, _I, _L, _P], _I),
    "nrcps_pair_matrix_ptrs": ([_P, _P, _P, _I, _L, _P, _P, _P], _I),
    "nrcps_slater_dets": ([_P, _P, _P, _I, _I, _I, _I, _P], _I),
    "nrcps_slater_dets_noalloc": ([_P, _P, _P, _I, _I, _I, _I, _P], _I),
    "nrcps_ensemble_create": ([_P, ctypes.POINTER(Job), _DP, _DP, _DP, _DP, _IP, _DP, _IP, ctypes.POINTER(_P)], _I),
    "nrcps_ensemble_run": ([_P, _U64, _P], _I),
    "nrcps_ensemble_set_sources": ([_P, _DP, _IP], _I),
    "nrcps_ensemble_destroy": ([_P], _I),
    "nrcps_ensemble_launches": ([_P, _LP], _I),
    "nrcps_ensemble_field_bits": ([_P, ctypes.POINTER(ctypes.c_void_p)], _I),
    "nrcps_accumulate": ([_P, _P, _I, _I, _I, _I, _I, _P, _P], _I),
    "nrcps_batch_create": ([_P, _P, _P, _I, ctypes.POINTER(_P)], _I),
    "nrcps_batch_output_size": ([_P, _LP, _LP], _I),
    "nrcps_batch_layout": ([_P, _I, _LP, _LP], _I),
    "nrcps_batch_run": ([_P, _P], _I),
    "nrcps_batch_destroy": ([_P], _I),
    "nrcps_shifted_pair_matrix": ([_P, _P, _P, _I, _I, _L, _I, _P, _P, _P, _I, _P], _I),
    "nrcps_branch_create": ([_P, _P, _P, _P, _P, _P, _P, ctypes.POINTER(_P)], _I),
    "nrcps_branch_run": ([_P, _P], _I),
    "nrcps_branch_destroy": ([_P], _I),
    "nrcps_cv_coarse_z2": ([_P, _P, _U64, _I, _I, _I, _I, _P], _I),
    "nrcps_cv_sample_z2_features": ([_P, _U64, _U64, _I, _I, _I, _I, _P], _I),
    "nrcps_reorthonormalise": ([_P, _P, _I, ctypes.c_long, _I, _I, _P, _P], _I),
    "nrcps_cv_forward_tc": ([_P, _P, _I, _I, _I, _P, _P, _P, _P, _I, _P, _P, _I, _P], _I),
    "nrcps_cv_conv_forward": ([_P, _P, _I, _I, _I, _I, _P, _P, _P, _P], _I),
    "nrcps_cv_conv_backward": ([_P, _P, _P, _P, _I, _I, _I, _I, _P, _P, _P, _P], _I),
    "nrcps_cv_head_forward": ([_P, _P, _I, _I, _I, _P, _P, _I, _P, _P, _I, _P, _P, _P], _I),
    "nrcps_cv_head_backward": ([_P, _P, _P, _I, _I, _P, _I, _P, _P, _I, _P, _I, _P, _P, _P, _P, _P, _P, _P, _P,
                                _P], _I),
    "nrcps_cv_adam": ([_P, _P, _P, _P, _P, _L, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, _I,
                       _P], _I),
    "nrcps_jackknife": ([_P, _P, _L, _I, _I, _P, _P, _P, _P], _I),
}

_lib = None


def lib() -> ctypes.CDLL:
    """Loads libnrcps_b200.so (building it first if it is absent)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from . import build as _build
            _build.build()
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def check(status: int, ctx=None, what: str = "") -> None:
    if status != OK:
        msg = lib().nrcps_last_error(ctx).decode() if ctx else ""
        raise NrcpsError(status, f"{what}: {msg}" if what else msg)
