"""ctypes binding of libbroccoli_b200.so (the C-ABI in include/broccoli_b200.h).

The shared library is built in-tree (``make -C broccoli_b200``) and loaded
from this directory.  There is no fallback: if the library is missing or no
sm_100 device is present the calls raise.
"""
from __future__ import annotations

import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbroccoli_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(HERE), "include", "broccoli_b200.h")

BRC_OK = 0
BRC_ERR_INVALID = -1
BRC_ERR_NOMEM = -2
BRC_ERR_CUDA = -3
BRC_ERR_TIMEOUT = -4
BRC_ERR_NODEVICE = -5
BRC_ERR_UNSUPPORTED = -6
BRC_ERR_NONFINITE = -7
BRC_ERR_SCRATCH_LIMIT = -8

TRANSLATION, RIGID, AFFINE = 0, 1, 2
PREC_FP32, PREC_BF16X3, PREC_FP32_GENERAL, PREC_TF32 = 0, 1, 2, 3
INTERP_NEAREST, INTERP_LINEAR, INTERP_CUBIC = 0, 1, 2


class BrcError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


class LinearOpts(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int),
        ("type", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("tolerance", ctypes.c_float),
        ("use_graph", ctypes.c_int),
        ("certainty_sigma_x100", ctypes.c_int),
    ]


class NonlinearOpts(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int),
        ("coarsest_scale", ctypes.c_int),
        ("tsigma", ctypes.c_float),
        ("esigma", ctypes.c_float),
        ("dsigma", ctypes.c_float),
        ("precision", ctypes.c_int),
        ("solve_fp64", ctypes.c_int),
    ]


class TwoVolumeOpts(ctypes.Structure):
    _fields_ = [
        ("linear_iterations", ctypes.c_int),
        ("nonlinear_iterations", ctypes.c_int),
        ("coarsest_scale", ctypes.c_int),
        ("mm_z_cut", ctypes.c_int),
        ("tsigma", ctypes.c_float),
        ("esigma", ctypes.c_float),
        ("dsigma", ctypes.c_float),
        ("precision", ctypes.c_int),
        ("solve_fp64", ctypes.c_int),
        ("precenter", ctypes.c_int),
    ]


class DebugOutputs(ctypes.Structure):
    _fields_ = [
        ("quadrature_responses", ctypes.c_void_p * 6),
        ("phase_differences", ctypes.c_void_p),
        ("phase_certainties", ctypes.c_void_p),
        ("phase_gradients", ctypes.c_void_p),
    ]


_F3 = ctypes.c_float * 3


class FirstLevelInput(ctypes.Structure):
    _fields_ = [
        ("fmri", ctypes.c_void_p),
        ("epi_w", ctypes.c_int), ("epi_h", ctypes.c_int), ("epi_d", ctypes.c_int), ("epi_t", ctypes.c_int),
        ("epi_voxel", _F3),
        ("t1", ctypes.c_void_p),
        ("t1_w", ctypes.c_int), ("t1_h", ctypes.c_int), ("t1_d", ctypes.c_int),
        ("t1_voxel", _F3),
        ("mni", ctypes.c_void_p),
        ("mni_w", ctypes.c_int), ("mni_h", ctypes.c_int), ("mni_d", ctypes.c_int),
        ("mni_voxel", _F3),
        ("filters3", ctypes.c_void_p),
        ("filters6", ctypes.c_void_p),
        ("tensors", ctypes.c_void_p),
        ("dirs", ctypes.c_void_p),
    ]


class FirstLevelOpts(ctypes.Structure):
    _fields_ = [
        ("linear_iterations", ctypes.c_int),
        ("nonlinear_iterations", ctypes.c_int),
        ("motion_iterations", ctypes.c_int),
        ("coarsest_scale_t1_mni", ctypes.c_int),
        ("coarsest_scale_epi_t1", ctypes.c_int),
        ("mm_t1_z_cut", ctypes.c_int),
        ("apply_motion_correction", ctypes.c_int),
        ("apply_smoothing", ctypes.c_int),
        ("smoothing_fwhm", ctypes.c_float),
        ("tsigma", ctypes.c_float),
        ("esigma", ctypes.c_float),
        ("dsigma", ctypes.c_float),
        ("precision", ctypes.c_int),
        ("solve_fp64", ctypes.c_int),
    ]


FIRST_LEVEL_OUTPUTS = ("params_t1_mni", "params_epi_t1", "params_epi_mni", "motion_parameters", "interpolated_t1",
                       "aligned_t1_linear", "aligned_t1_nonlinear", "field", "aligned_epi_t1",
                       "aligned_epi_mni_linear", "aligned_epi_mni_nonlinear", "motion_corrected", "epi_mask",
                       "smoothed")


class FirstLevelOutput(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in FIRST_LEVEL_OUTPUTS]


_lib = None

_P = ctypes.c_void_p
_I = ctypes.c_int
_LL = ctypes.c_longlong

_SIGS = {
    "brc_version": ([], ctypes.c_char_p),
    "brc_status_string": ([_I], ctypes.c_char_p),
    "brc_last_error": ([_P], ctypes.c_char_p),
    "brc_ctx_create": ([_I, ctypes.POINTER(_P)], _I),
    "brc_ctx_destroy": ([_P], _I),
    "brc_ctx_set_stream": ([_P, _P], _I),
    "brc_ctx_stream": ([_P], _P),
    "brc_ctx_synchronize": ([_P], _I),
    "brc_selftest_bounded_wait": ([_P, _I], _I),
    "brc_selftest_phase_atan2": ([_P, _P, _P, _P, _LL], _I),
    "brc_ctx_workspace_bytes": ([_P], ctypes.c_size_t),
    "brc_ctx_kernel_launches": ([_P], ctypes.c_ulonglong),
    "brc_filter3d": ([_P, _P, _I, _I, _I, _I, _LL, _P, _I, _I, _P], _I),
    "brc_normal_equations": ([_P, _P, _LL, _P, _I, _I, _I, _I, _P, _P], _I),
    "brc_solve_affine_fp64": ([_P, _P, _P, _I, _P], _I),
    "brc_warp_affine": ([_P, _P, _I, _I, _I, _I, _P, _P], _I),
    "brc_warp_field": ([_P, _P, _I, _I, _I, _P, _P, _P, _P], _I),
    "brc_smooth3d": ([_P, _P, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P], _I),
    "brc_smooth_normalized": ([_P, _P, _I, _I, _I, _I, _P, _P, _P, _P, _P], _I),
    "brc_rescale_linear": ([_P, _P, _I, _I, _I, _P, _I, _I, _I], _I),
    "brc_linear_opts_default": ([ctypes.POINTER(LinearOpts), _I], None),
    "brc_register_linear_batched": (
        [_P, _P, _LL, _P, _I, _I, _I, _I, _P, ctypes.POINTER(LinearOpts), _P, _P, _P, _P], _I),
    "brc_motion_correct": (
        [_P, _P, _I, _I, _I, _I, _P, _P, ctypes.POINTER(LinearOpts), _P, _P], _I),
    "brc_register_linear_scales": (
        [_P, _P, _P, _I, _I, _I, _I, _P, ctypes.POINTER(LinearOpts), _I, _P, _P, _P], _I),
    "brc_nonlinear_opts_default": ([ctypes.POINTER(NonlinearOpts), _I], None),
    "brc_nonlinear_step": (
        [_P, _P, _P, _I, _I, _I, _P, _P, ctypes.c_float, ctypes.c_float, ctypes.c_float, _I, _P], _I),
    "brc_register_nonlinear": (
        [_P, _P, _P, _I, _I, _I, _P, _P, _P, ctypes.POINTER(NonlinearOpts), _P, _P], _I),
    "brc_change_resolution_and_size": ([_P, _P, _I, _I, _I, _P, _P, _I, _I, _I, _P, _I], _I),
    "brc_center_of_mass": ([_P, _P, _I, _I, _I, _P], _I),
    "brc_change_resolution_and_size_batch": ([_P, _P, _I, _I, _I, _I, _P, _P, _I, _I, _I, _P, _I, _I], _I),
    "brc_transform_volumes_linear": ([_P, _P, _I, _I, _I, _I, _P, _I, _P], _I),
    "brc_transform_volumes_nonlinear": ([_P, _P, _I, _I, _I, _I, _P, _P, _P, _I, _P], _I),
    "brc_combine_displacement_field": ([_P, _P, _P, _P, _I, _I, _I, _P], _I),
    "brc_center_volumes": ([_P, _P, _I, _I, _I, _I, _I, _P, _P], _I),
    "brc_two_volume_opts_default": ([ctypes.POINTER(TwoVolumeOpts)], None),
    "brc_register_two_volumes": (
        [_P, _P, _I, _I, _I, _P, _P, _I, _I, _I, _P, _P, _P, _P, _P, ctypes.POINTER(TwoVolumeOpts), _P, _P,
         _P, _P, _P], _I),
    "brc_smoothing_filters_fwhm": ([ctypes.c_float, _P, _P, _P, _P], None),
    "brc_tensor_magnitude": ([_P, _P, _I, _I, _I, _P, _P, _I, _P], _I),
    "brc_segment_epi": ([_P, _P, _I, _I, _I, _P, _P], _I),
    "brc_first_level_opts_default": ([ctypes.POINTER(FirstLevelOpts)], None),
    "brc_first_level_preprocess": ([_P, ctypes.POINTER(FirstLevelInput), ctypes.POINTER(FirstLevelOpts),
                                    ctypes.POINTER(FirstLevelOutput)], _I),
    "brc_ctx_set_debug_outputs": ([_P, ctypes.POINTER(DebugOutputs)], _I),
    "brc_phase_volumes": ([_P, _P, _P, _I, _I, _I, _I, _P, _P, _P], _I),
    "brc_multiply_volumes": ([_P, _P, _I, _I, _I, _I, _P], _I),
    "brc_invert_affine_parameters": ([_P, _P], None),
    "brc_register_cohort": (
        [_P, _I, _P, _P, _P, _P, _I, _I, _I, _P, _P, _P, _P, _P, ctypes.POINTER(TwoVolumeOpts), _P, _P, _P, _P],
        _I),
}


def header_symbols(path: str = HEADER_PATH) -> list:
    """Function names declared in the C-ABI header."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(brc_[a-z0-9_]+)\s*\(", text)))


def lib():
    """The loaded library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {HERE}` "
                               "or __graft_entry__.build()")
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def status_string(s: int) -> str:
    return lib().brc_status_string(s).decode()
