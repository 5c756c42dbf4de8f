"""Loader of libgfft.so and the status -> exception mapping.

The sentinel exceptions mirror errors.go:6-30 of the reference, so code
written against the Go API (``errors.Is(err, ErrLengthMismatch)``) maps to
``except ErrLengthMismatch``.
"""
from __future__ import annotations

import ctypes
import os

_PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.environ.get("GFFT_LIB", os.path.join(_PKG_DIR, "libgfft.so"))

_lib = None


class GfftError(RuntimeError):
    status = -1


class ErrInvalidLength(GfftError):
    status = 1


class ErrNilSlice(GfftError):
    status = 2


class ErrLengthMismatch(GfftError):
    status = 3


class ErrInvalidStride(GfftError):
    status = 4


class ErrInvalidSpectrum(GfftError):
    status = 5


class ErrNotImplemented(GfftError):
    status = 6


class ErrCuda(GfftError):
    status = 100


class ErrOutOfMemory(GfftError):
    status = 101


class ErrTimeout(GfftError):
    status = 102


class ErrNoDevice(GfftError):
    status = 103


class ErrInvalidArgument(GfftError):
    status = 104


class ErrWisdom(GfftError):
    status = 105


_BY_STATUS = {c.status: c for c in (ErrInvalidLength, ErrNilSlice, ErrLengthMismatch, ErrInvalidStride,
                                    ErrInvalidSpectrum, ErrNotImplemented, ErrCuda, ErrOutOfMemory, ErrTimeout,
                                    ErrNoDevice, ErrInvalidArgument, ErrWisdom)}

# (name, restype, argtypes) of every exported entry point of include/gfft.h.
P = ctypes.c_void_p
I32 = ctypes.c_int32
I64 = ctypes.c_int64
SZ = ctypes.c_size_t
CHARP = ctypes.c_char_p
PP = ctypes.POINTER(ctypes.c_void_p)


class PlanOptionsC(ctypes.Structure):
    _fields_ = [("planner", I32), ("strategy", I32), ("batch", I64), ("stride", I64), ("in_place", I32),
                ("device", I32)]


SIGNATURES = {
    "gfft_plan_new": (I32, [PP, I32, I64, ctypes.POINTER(PlanOptionsC)]),
    "gfft_plan_close": (None, [P]),
    "gfft_plan_len": (I64, [P]),
    "gfft_plan_algorithm": (I32, [P, CHARP, SZ]),
    "gfft_plan_new_variant": (I32, [PP, I32, I64, CHARP]),
    "gfft_plan_variants": (I32, [I32, I64, CHARP, SZ, ctypes.POINTER(SZ)]),
    "gfft_plan_check": (I32, [P]),
    "gfft_autotune": (I32, [I32, I64, I64, I32, CHARP, SZ, ctypes.POINTER(SZ)]),
    "gfft_wisdom_import_string": (I32, [CHARP]),
    "gfft_wisdom_export_string": (I32, [CHARP, SZ, ctypes.POINTER(SZ)]),
    "gfft_wisdom_import_file": (I32, [CHARP]),
    "gfft_wisdom_export_file": (I32, [CHARP]),
    "gfft_wisdom_clear": (None, []),
    "gfft_wisdom_len": (I64, []),
    "gfft_forward": (I32, [P, P, I64, P, I64, P]),
    "gfft_inverse": (I32, [P, P, I64, P, I64, P]),
    "gfft_forward_batch": (I32, [P, P, I64, P, I64, I64, P]),
    "gfft_inverse_batch": (I32, [P, P, I64, P, I64, I64, P]),
    "gfft_forward_strided": (I32, [P, P, I64, P, I64, I64, P]),
    "gfft_inverse_strided": (I32, [P, P, I64, P, I64, I64, P]),
    "gfft_exec_batch_noalloc": (I32, [P, I32, P, I64, P, I64, I64, P]),
    "gfft_forward_host": (I32, [P, P, I64, P, I64]),
    "gfft_inverse_host": (I32, [P, P, I64, P, I64]),
    "gfft_forward_batch_host": (I32, [P, P, I64, P, I64, I64]),
    "gfft_inverse_batch_host": (I32, [P, P, I64, P, I64, I64]),
    "gfft_plan_real_new": (I32, [PP, I32, I64, ctypes.POINTER(PlanOptionsC)]),
    "gfft_plan_real_close": (None, [P]),
    "gfft_plan_real_len": (I64, [P]),
    "gfft_plan_real_spectrum_len": (I64, [P]),
    "gfft_real_forward": (I32, [P, I32, P, I64, P, I64, P]),
    "gfft_real_inverse": (I32, [P, P, I64, P, I64, P]),
    "gfft_real_forward_host": (I32, [P, I32, P, I64, P, I64]),
    "gfft_real_inverse_host": (I32, [P, P, I64, P, I64]),
    "gfft_plan_nd_new": (I32, [PP, I32, I32, ctypes.POINTER(I64), I32, ctypes.POINTER(PlanOptionsC)]),
    "gfft_plan_nd_close": (None, [P]),
    "gfft_plan_nd_len": (I64, [P]),
    "gfft_plan_nd_spectrum_len": (I64, [P]),
    "gfft_nd_forward": (I32, [P, P, I64, P, I64, P]),
    "gfft_nd_inverse": (I32, [P, P, I64, P, I64, P]),
    "gfft_nd_forward_full": (I32, [P, P, I64, P, I64, P]),
    "gfft_nd_inverse_full": (I32, [P, P, I64, P, I64, P]),
    "gfft_nd_forward_host": (I32, [P, P, I64, P, I64]),
    "gfft_nd_inverse_host": (I32, [P, P, I64, P, I64]),
    "gfft_exec_strided_batch": (I32, [P, I32, P, I64, P, I64, I64, I64, I64, P]),
    "gfft_convolve": (I32, [I32, P, I64, P, I64, P, I64, P]),
    "gfft_correlate": (I32, [I32, P, I64, P, I64, P, I64, P]),
    "gfft_convolve_real": (I32, [I32, P, I64, P, I64, P, I64, P]),
    "gfft_convolve_host": (I32, [I32, P, I64, P, I64, P, I64]),
    "gfft_correlate_host": (I32, [I32, P, I64, P, I64, P, I64]),
    "gfft_convolve_real_host": (I32, [I32, P, I64, P, I64, P, I64]),
    "gfft_convolve_real_batch": (I32, [I32, P, I64, P, I64, I64, I64, P, I64, P]),
    "gfft_plan_uneven_new": (I32, [PP, I32, I64, ctypes.POINTER(I64), ctypes.POINTER(PlanOptionsC)]),
    "gfft_plan_uneven_close": (None, [P]),
    "gfft_plan_uneven_total": (I64, [P]),
    "gfft_uneven_exec": (I32, [P, I32, P, P, I32, P]),
    "gfft_uneven_exec_per_size": (I32, [P, I32, P, P, P]),
    "gfft_mlp_sizes": (None, [ctypes.POINTER(I32), ctypes.POINTER(I32), ctypes.POINTER(I64)]),
    "gfft_mlp_forward": (I32, [P, P, I64, P, P]),
    "gfft_mlp_grad": (I32, [P, P, P, I64, P, P, P]),
    "gfft_mlp_train": (I32, [P, P, P, P, P, I64, I32, I32, ctypes.c_float, ctypes.c_uint64, I64, P, P]),
    "gfft_planner_features": (I32, [I32, I64, I64, I64, I32, CHARP, P]),
    "gfft_planner_set_model": (I32, [P, P]),
    "gfft_planner_load_model": (I32, [CHARP]),
    "gfft_planner_has_model": (I32, []),
    "gfft_planner_choose": (I32, [I32, I64, I64, I64, I32, ctypes.c_char_p, ctypes.c_size_t]),
    "gfft_plan_clone": (I32, [PP, P]),
    "gfft_plan_new_pooled": (I32, [PP, I32, I64, ctypes.POINTER(PlanOptionsC)]),
    "gfft_plan_pool_clear": (None, []),
    "gfft_set_kernel_strategy": (None, [I32]),
    "gfft_get_kernel_strategy": (I32, []),
    "gfft_record_benchmark_decision": (None, [I64, I32]),
    "gfft_status_string": (CHARP, [I32]),
    "gfft_last_error": (CHARP, []),
    "gfft_device_count": (I32, [ctypes.POINTER(I32)]),
    "gfft_buffer_alloc": (I32, [PP, I64]),
    "gfft_buffer_free": (I32, [P]),
    "gfft_buffer_upload": (I32, [P, P, I64]),
    "gfft_buffer_download": (I32, [P, P, I64]),
    "gfft_stream_create": (I32, [PP]),
    "gfft_stream_synchronize": (I32, [P]),
    "gfft_stream_destroy": (I32, [P]),
}


def lib():
    """Loads libgfft.so (raising if it has not been built: there is no CPU
    fallback) and declares every signature."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libgfft.so not built at {LIB_PATH}; run algo-fft_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status == 0:
        return
    L = lib()
    detail = (L.gfft_last_error() or b"").decode()
    text = (L.gfft_status_string(status) or b"").decode()
    cls = _BY_STATUS.get(status, GfftError)
    raise cls(f"{text}: {detail}" if detail else text)
