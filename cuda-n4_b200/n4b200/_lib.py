"""ctypes binding of the C ABI declared in ``include/n4b200.h``.

Loading fails loudly when ``libn4b200.so`` has not been built: there is no
CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os

N4_MAX_LEVELS = 8

N4_OK = 0
STATUS = {
    0: "N4_OK", 1: "N4_ERR_INVALID_ARG", 2: "N4_ERR_UNSUPPORTED_SPLINE_ORDER",
    3: "N4_ERR_EMPTY_MASK", 4: "N4_ERR_OOM", 5: "N4_ERR_CUDA", 6: "N4_ERR_TIMEOUT",
    7: "N4_ERR_NONFINITE", 8: "N4_ERR_TOO_LARGE", 9: "N4_ERR_NO_DEVICE",
}

FLAG_CV_DDOF1 = 0x1
FLAG_CTA_512 = 0x2000
FLAG_MASK_U8 = 0x4000
FLAG_FIT_ZERO_DEN = 0x2
FLAG_INPLACE_THRESH = 0x4
FLAG_FORCE_GRID = 0x8
FLAG_FORCE_CLUSTER = 0x10


def FLAG_SUB_BATCHES(k: int) -> int:
    """Bits 16-18 of n4_params_t.flags: k sub-batches (0 = automatic, 1 = no overlap)."""
    return (int(k) & 7) << 16


def FLAG_SUB_CLUSTER_FLOOR(k: int) -> int:
    """Bits 19-23 of n4_params_t.flags: with two or more sub-batches, each on
    the smallest cluster size >= k that holds its volumes (0 = one size)."""
    return (int(k) & 31) << 19


class n4_params_t(C.Structure):
    _fields_ = [
        ("NumberOfHistogramBins", C.c_uint),
        ("WienerFilterNoise", C.c_float),
        ("BiasFieldFullWidthAtHalfMaximum", C.c_float),
        ("NumberOfControlPoints_x", C.c_uint),
        ("NumberOfControlPoints_y", C.c_uint),
        ("NumberOfControlPoints_z", C.c_uint),
        ("NumberOfFittingLevels", C.c_uint),
        ("MaximumNumberOfIterations", C.c_uint * N4_MAX_LEVELS),
        ("ConvergenceThreshold", C.c_float),
        ("low_value", C.c_float),
        ("ShrinkFactor", C.c_uint),
        ("SplineOrder", C.c_uint),
        ("FitEpsilon", C.c_float),
        ("flags", C.c_uint),
    ]


class n4_report_t(C.Structure):
    _fields_ = [
        ("status", C.c_int),
        ("levels", C.c_int),
        ("iterations", C.c_int * N4_MAX_LEVELS),
        ("final_cv", C.c_float * N4_MAX_LEVELS),
        ("warm_start_used", C.c_int),
        ("first_cv_warm", C.c_float),
        ("first_cv_plain", C.c_float),
        ("foreground", C.c_longlong),
        ("path", C.c_int),
        ("cluster_size", C.c_int),
        ("device_begin_ns", C.c_ulonglong),
        ("device_end_ns", C.c_ulonglong),
        ("sm", C.c_int),
        ("reserved", C.c_int),
    ]


class n4_volume_t(C.Structure):
    _fields_ = [
        ("im", C.c_void_p), ("mask", C.c_void_p),
        ("fx", C.c_uint), ("fy", C.c_uint), ("fz", C.c_uint),
        ("im_normalized", C.c_void_p), ("lattice", C.c_void_p),
        ("bias_field", C.c_void_p), ("warm_lattice", C.c_void_p),
    ]


N4_TUNE_MAX = 24


class n4_tune_report_t(C.Structure):
    _fields_ = [
        ("candidates", C.c_int), ("cluster_size", C.c_int * N4_TUNE_MAX), ("threads", C.c_int * N4_TUNE_MAX),
        ("ms", C.c_float * N4_TUNE_MAX),
        ("chosen", C.c_int),
        ("corr_candidates", C.c_int), ("corr_rows", C.c_int * N4_TUNE_MAX),
        ("corr_threads", C.c_int * N4_TUNE_MAX), ("corr_ms", C.c_float * N4_TUNE_MAX), ("corr_chosen", C.c_int),
        ("sub_candidates", C.c_int), ("sub_count", C.c_int * N4_TUNE_MAX), ("sub_tapered", C.c_int * N4_TUNE_MAX),
        ("sub_ms", C.c_float * N4_TUNE_MAX), ("sub_chosen", C.c_int), ("sub_adapt", C.c_int * N4_TUNE_MAX),
    ]


class n4_component_tune_t(C.Structure):
    _fields_ = [
        ("fit_candidates", C.c_int), ("fit_step", C.c_int * N4_TUNE_MAX), ("fit_depth", C.c_int * N4_TUNE_MAX),
        ("fit_rows", C.c_int * N4_TUNE_MAX), ("fit_ms", C.c_float * N4_TUNE_MAX), ("fit_chosen", C.c_int),
        ("fit_shape", C.c_int),
        ("eval_candidates", C.c_int), ("eval_rows", C.c_int * N4_TUNE_MAX), ("eval_threads", C.c_int * N4_TUNE_MAX),
        ("eval_ms", C.c_float * N4_TUNE_MAX), ("eval_chosen", C.c_int), ("eval_shape", C.c_int),
    ]


class n4_timings_t(C.Structure):
    _fields_ = [
        ("stage_ms", C.c_float * 4), ("launches", C.c_int), ("fit_voxels", C.c_longlong),
        ("full_voxels", C.c_longlong),
        ("fit_rows", C.c_int), ("fit_step", C.c_int), ("fit_depth", C.c_int), ("reserved", C.c_int),
        ("correct_rows", C.c_int), ("correct_threads", C.c_int),
    ]


LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libn4b200.so")

# (name, restype, argtypes) of every exported entry point of include/n4b200.h
_P = C.c_void_p
_U = C.c_uint
SIGNATURES = [
    ("n4_params_default", None, [C.POINTER(n4_params_t)]),
    ("n4_lattice_dims", C.c_int, [C.POINTER(n4_params_t), C.POINTER(C.c_uint), C.POINTER(C.c_size_t)]),
    ("n4_fitting_dims", C.c_int, [C.POINTER(n4_params_t), C.c_uint, C.c_uint, C.c_uint, C.POINTER(C.c_uint)]),
    ("n4_status_string", C.c_char_p, [C.c_int]),
    ("n4_last_error_string", C.c_char_p, []),
    ("n4_version", C.c_char_p, []),
    ("n4_create", C.c_int, [C.POINTER(C.c_void_p), C.c_int]),
    ("n4_destroy", C.c_int, [_P]),
    ("n4_run", C.c_int, [_P, C.POINTER(n4_params_t), _P, _P, _U, _U, _U, _P, _P, _P, _P, _P,
                         C.POINTER(n4_report_t)]),
    ("n4_run_host", C.c_int, [_P, C.POINTER(n4_params_t), _P, _P, _U, _U, _U, _P, _P, _P, _P,
                              C.POINTER(n4_report_t)]),
    ("n4_run_batched", C.c_int, [_P, C.POINTER(n4_params_t), C.c_int, C.POINTER(n4_volume_t), _P,
                                 C.POINTER(n4_report_t)]),
    ("n4_sync", C.c_int, [_P, C.POINTER(n4_report_t), C.c_int]),
    ("n4_batch_graph_create", C.c_int, [_P, C.POINTER(n4_params_t), C.c_int, C.POINTER(n4_volume_t),
                                        C.POINTER(C.c_void_p)]),
    ("n4_batch_graph_launch", C.c_int, [_P, _P]),
    ("n4_batch_graph_sync", C.c_int, [_P, C.POINTER(n4_report_t), C.c_int]),
    ("n4_batch_graph_destroy", C.c_int, [_P]),
    ("n4_batch_graph_info", C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("n4_set_profiling", C.c_int, [_P, C.c_int]),
    ("n4_last_timings", C.c_int, [_P, C.POINTER(n4_timings_t)]),
    ("n4_autotune", C.c_int, [_P, _P, C.c_int, _P, _P, _P]),
    ("n4_run_batched_host", C.c_int, [_P, _P, C.c_int, _P, C.c_int, _P, _P, C.POINTER(C.c_float)]),
    ("n4_autotune_components", C.c_int, [_P, _P, _P, C.c_uint, C.c_uint, C.c_uint, C.c_uint, C.c_uint, C.c_uint,
                                         _P, _P, _P, _P]),
    ("n4_warm_inputs", C.c_int, [_P, _P, C.c_int, _P, _P, _P]),
    ("n4_run_batched_warm", C.c_int, [_P, _P, C.c_int, _P, _P, _P, _P]),
    ("n4_batch_graph_create_warm", C.c_int, [_P, _P, C.c_int, _P, _P, _P]),
    ("n4_fit_bspline3d", C.c_int, [_P, _P, _P, _U, _U, _U, _U, _U, _U, C.c_float, C.c_int, _P, _P]),
    ("n4_fit_bspline3d_noalloc", C.c_int, [_P, _P, _U, _U, _U, _U, _U, _U, C.c_float, C.c_int, _P, _P]),
    ("n4_evaluate_bspline3d", C.c_int, [_P, _P, _U, _U, _U, _U, _U, _U, _P, _P]),
    ("n4_upsample_lattice3d", C.c_int, [_P, _P, _U, _U, _U, _P, _P]),
    ("n4_sharpen_image", C.c_int, [_P, _P, _P, _U, _U, C.c_float, C.c_float, _P,
                                   C.POINTER(C.c_float), C.POINTER(C.c_float), _P]),
    ("n4_convergence", C.c_int, [_P, _P, _P, _P, _U, C.c_int, C.POINTER(C.c_double)]),
    ("n4_encoder_num_params", C.c_size_t, []),
    ("n4_encoder_create", C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.c_int]),
    ("n4_encoder_destroy", C.c_int, [_P]),
    ("n4_encoder_set_params", C.c_int, [_P, _P, C.c_size_t]),
    ("n4_encoder_get_params", C.c_int, [_P, _P, _P, C.c_size_t]),
    ("n4_encoder_predict", C.c_int, [_P, _P, C.c_int, _P, _P]),
    ("n4_encoder_train_step", C.c_int, [_P, _P, _P, C.c_int, C.c_float, C.POINTER(C.c_float), _P]),
]

_lib = None


def load(path: str = LIB_PATH):
    """Load the library (once) and declare every entry point."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with `python cuda-n4_b200/n4b200/build.py` "
            "(n4b200 has no CPU fallback)")
    lib = C.CDLL(path)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class N4Error(RuntimeError):
    def __init__(self, status: int, message: str = ""):
        self.status = status
        super().__init__(f"{STATUS.get(status, status)}: {message}")


def check(status: int):
    if status != N4_OK:
        msg = load().n4_last_error_string().decode(errors="replace")
        raise N4Error(status, msg)
