"""ctypes binding of ``libhuv_b200.so`` (the C ABI of include/huv_b200.h).

Loading fails loudly when the library has not been built: there is no
Python or CPU fallback for any imaging call.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhuv_b200.so")

HUV_OK = 0
STATUS_NAMES = {
    0: "OK", 1: "INVALID_PARAMETER", 2: "GRID_NOT_POWER_OF_TWO", 3: "NO_DIFFRACTION_ORDERS",
    4: "PUPIL_SAMPLING_TOO_DENSE", 5: "TCC_DECOMPOSITION", 6: "DIMENSION_MISMATCH", 7: "NUMERICAL",
    8: "CUDA", 9: "OUT_OF_MEMORY", 10: "DEVICE_TIMEOUT", 11: "UNSUPPORTED",
}

FILL = {"conventional": 0, "annular": 1, "quadrupole": 2, "dipole": 3, "gaussian": 4, "quasar": 5}
OPTICS_PROJECTION, OPTICS_EUV = 0, 1
INPUT_U8, INPUT_F32, INPUT_C64, INPUT_RECTS = 0, 1, 2, 3
FORM = {"auto": 0, "fft": 1, "tc": 2, "tc_rows": 3, "hybrid": 4}


class HuvError(RuntimeError):
    """A non-OK huv_status; ``status`` holds the code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class Source(C.Structure):
    _fields_ = [("wavelength_nm", C.c_double), ("fill", C.c_int32), ("p", C.c_double * 4)]


class Optics(C.Structure):
    _fields_ = [("kind", C.c_int32), ("na", C.c_double), ("flare_fraction", C.c_double),
                ("immersion_index", C.c_double), ("central_obscuration", C.c_double),
                ("transmission", C.c_double), ("paraxial_defocus", C.c_int32)]


class Grid(C.Structure):
    _fields_ = [("size", C.c_int32), ("pixel_nm", C.c_double)]


class Settings(C.Structure):
    _fields_ = [("max_kernels", C.c_int32), ("kernel_energy_fraction", C.c_double),
                ("source_points_per_axis", C.c_int32), ("normalization", C.c_int32),
                ("kernel_cache_capacity", C.c_int32), ("kernel_build", C.c_int32)]


class Diagnostics(C.Structure):
    _fields_ = [("num_kernels", C.c_int32), ("captured_energy_fraction", C.c_double),
                ("num_frequencies", C.c_int32), ("num_columns", C.c_int32), ("method", C.c_int32),
                ("support_exceeds_nyquist", C.c_int32), ("clear_field_intensity", C.c_double),
                ("normalized", C.c_int32), ("band_half_width", C.c_int32),
                ("num_source_points", C.c_int32)]


class KernelSetDesc(C.Structure):
    """huv_kernel_set."""
    _fields_ = [("grid_size", C.c_int32), ("pixel_nm", C.c_double), ("n_kernels", C.c_int32),
                ("eigenvalues", C.c_void_p), ("kernels", C.c_void_p), ("defocus_nm", C.c_double),
                ("wavelength_nm", C.c_double), ("captured_energy_fraction", C.c_double),
                ("flare_fraction", C.c_double)]


class Clip(C.Structure):
    _fields_ = [("engine", C.c_void_p), ("max_kernels", C.c_int32), ("input_kind", C.c_int32),
                ("input", C.c_void_p), ("out", C.c_void_p)]


class IltParams(C.Structure):
    _fields_ = [("cost_kind", C.c_int32), ("threshold", C.c_double), ("steepness", C.c_double),
                ("beta", C.c_double), ("tv_weight", C.c_double), ("tv_epsilon", C.c_double),
                ("binarization_weight", C.c_double), ("dose", C.c_double), ("weight", C.c_double),
                ("absorber", C.c_double), ("defocus_nm", C.c_double)]


class IltOpt(C.Structure):
    _fields_ = [("max_iterations", C.c_int32), ("learning_rate", C.c_double), ("convergence_tol", C.c_double)]


class SurrogateIlt(C.Structure):
    _fields_ = [("judge_every", C.c_int32), ("error_bound", C.c_double), ("surrogate_iterations", C.c_int32),
                ("exact_iterations", C.c_int32), ("takeover_iteration", C.c_int32), ("n_judges", C.c_int32),
                ("judge_errors", C.c_double * 64)]


class Rect(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("w", C.c_double), ("h", C.c_double)]


class RectClips(C.Structure):
    _fields_ = [("rects", C.c_void_p), ("offsets", C.c_void_p), ("feature_re", C.c_double),
                ("feature_im", C.c_double), ("background_re", C.c_double), ("background_im", C.c_double)]


class Batch(C.Structure):
    _fields_ = [("n_clips", C.c_int32), ("input_kind", C.c_int32), ("input", C.c_void_p),
                ("pixel_transfer", C.c_int32), ("defocus_nm", C.c_double), ("form", C.c_int32),
                ("eval_grid", C.c_int32)]


_lib = None

# Every entry point declared in include/huv_b200.h with its ctypes signature.
SIGNATURES = {
    "huv_last_error": (C.c_char_p, []),
    "huv_version": (C.c_char_p, []),
    "huv_engine_create": (C.c_int, [C.POINTER(Source), C.POINTER(Optics), C.POINTER(Grid),
                                    C.POINTER(Settings), C.c_int32, C.POINTER(C.c_void_p)]),
    "huv_engine_destroy": (None, [C.c_void_p]),
    "huv_kernelset_create": (C.c_int, [C.POINTER(KernelSetDesc), C.c_int32, C.POINTER(C.c_void_p)]),
    "huv_engine_source_points": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]),
    "huv_engine_diagnostics": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(Diagnostics)]),
    "huv_engine_clear_field": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(C.c_double)]),
    "huv_engine_kernels": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_int32,
                                     C.POINTER(C.c_int32)]),
    "huv_image_batch": (C.c_int, [C.c_void_p, C.POINTER(Batch), C.c_void_p, C.c_void_p]),
    "huv_image_batch_host": (C.c_int, [C.c_void_p, C.POINTER(Batch), C.c_void_p, C.c_void_p]),
    "huv_rasterize_rects": (C.c_int, [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32,
                                      C.c_void_p, C.c_void_p]),
    "huv_device_status": (C.c_int, [C.c_void_p, C.c_void_p]),
    "huv_debug_probe_wait": (C.c_int, [C.c_int64]),
    "huv_fno_create": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_uint64, C.c_int32,
                                 C.POINTER(C.c_void_p)]),
    "huv_fno_destroy": (None, [C.c_void_p]),
    "huv_fno_params": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(C.c_int64)]),
    "huv_fno_set_params": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64]),
    "huv_fno_forward": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "huv_fno_backward": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.POINTER(C.c_float), C.c_void_p]),
    "huv_fno_train_step": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_float, C.c_float,
                                     C.POINTER(C.c_float), C.c_void_p]),
    "huv_fno_device_status": (C.c_int, [C.c_void_p, C.c_void_p]),
    "huv_plan_create": (C.c_int, [C.POINTER(Clip), C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]),
    "huv_plan_launch": (C.c_int, [C.c_void_p, C.c_void_p]),
    "huv_plan_describe": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int32]),
    "huv_plan_destroy": (None, [C.c_void_p]),
    "huv_ilt_cost_grad": (C.c_int, [C.c_void_p, C.POINTER(IltParams), C.c_int32, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_void_p]),
    "huv_ilt_optimize": (C.c_int, [C.c_void_p, C.POINTER(IltParams), C.POINTER(IltOpt), C.c_int32, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "huv_ilt_optimize_surrogate": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(IltParams), C.POINTER(IltOpt),
                                             C.c_int32, C.c_void_p, C.c_void_p, C.POINTER(SurrogateIlt),
                                             C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "huv_image_focus_sweep": (C.c_int, [C.c_void_p, C.POINTER(Batch), C.c_void_p, C.c_int32, C.c_void_p,
                                        C.c_void_p]),
    "huv_image_batch_noalloc": (C.c_int, [C.c_void_p, C.POINTER(Batch), C.c_void_p, C.c_void_p]),
    "huv_profile_enable": (C.c_int, [C.c_void_p, C.c_int32]),
    "huv_profile_regions": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int32]),
    "huv_profile_read": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int32),
                                   C.POINTER(C.c_int64), C.c_char_p, C.c_int32]),
}


def lib():
    """The loaded library (raises if it was never built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m highuvlith_b200.build` "
                "(there is no fallback implementation)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != HUV_OK:
        msg = lib().huv_last_error()
        raise HuvError(status, msg.decode() if msg else "")
