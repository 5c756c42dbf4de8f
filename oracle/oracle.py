"""ctypes wrapper of the CPU oracle.  TEST INFRASTRUCTURE ONLY.

Only the tests, the smoke check and the benchmark's CPU-baseline leg import
this module; the product library never does.  ``liboracle.so`` is built from
``oracle.cpp`` by ``oracle/Makefile`` (``build()`` in ``__graft_entry__``
runs it).  The C++ file cites, per function, the reference file:line it
restates.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

# Reference strategy ids returned by orc_algorithm (plan.go:343-368).
ALGO_DIT, ALGO_STOCKHAM, ALGO_SIXSTEP, ALGO_MIXED, ALGO_BLUESTEIN = range(5)


def build(force: bool = False) -> str:
    src = os.path.join(_HERE, "oracle.cpp")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-C", _HERE, "-B" if force else "-s"], check=True,
                       stdout=subprocess.DEVNULL)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        I64 = ctypes.c_int64
        I = ctypes.c_int
        L.orc_naive_dft_f64.argtypes = [P, P, I64, I]
        L.orc_naive_dft_ref.argtypes = [P, P, I64, I]
        L.orc_naive_dft_nd_ref.argtypes = [P, P, I, P, I]
        L.orc_naive_dft_nd_f64.argtypes = [P, P, I, P, I]
        L.orc_algorithm.argtypes = [I64]
        L.orc_batch_c64.argtypes = [P, P, I64, I64, I, I]
        L.orc_batch_c128.argtypes = [P, P, I64, I64, I, I]
        L.orc_transform_algo_c64.argtypes = [P, P, I64, I, I]
        L.orc_real_forward_f32.argtypes = [P, P, I64, I64, I]
        L.orc_real_inverse_f32.argtypes = [P, P, I64, I64, I]
        L.orc_real_forward_f64.argtypes = [P, P, I64, I64]
        L.orc_real_inverse_f64.argtypes = [P, P, I64, I64]
        L.orc_convolve_real_f32.argtypes = [P, P, I64, P, I64]
        L.orc_convolve_c64.argtypes = [P, P, I64, P, I64]
        L.orc_twiddles_c64.argtypes = [P, I64]
        L.orc_twiddles_c128.argtypes = [P, I64]
        for name in ("orc_algorithm", "orc_batch_c64", "orc_batch_c128", "orc_transform_algo_c64",
                     "orc_real_forward_f32", "orc_real_inverse_f32", "orc_real_forward_f64",
                     "orc_real_inverse_f64", "orc_convolve_real_f32", "orc_convolve_c64",
                     "orc_max_threads"):
            getattr(L, name).restype = I
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def naive_dft(x: np.ndarray, inverse: bool = False) -> np.ndarray:
    """FP64 arbiter (exact angle reduction); returns complex128."""
    x = np.ascontiguousarray(x, dtype=np.complex128)
    y = np.empty_like(x)
    lib().orc_naive_dft_f64(_p(x), _p(y), x.size, int(inverse))
    return y


def naive_dft_ref(x: np.ndarray, inverse: bool = False) -> np.ndarray:
    """The reference oracle's own formula (internal/reference/dft.go)."""
    x = np.ascontiguousarray(x, dtype=np.complex128)
    y = np.empty_like(x)
    lib().orc_naive_dft_ref(_p(x), _p(y), x.size, int(inverse))
    return y


def _nd(fn, x: np.ndarray, dims, inverse: bool) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.complex128).ravel()
    d = np.ascontiguousarray(np.asarray(dims, dtype=np.int64))
    if int(np.prod(d)) != x.size:
        raise ValueError("input length must equal the product of the dimensions")
    y = np.empty_like(x)
    fn(_p(x), _p(y), int(d.size), _p(d), int(inverse))
    return y


def naive_dft_nd(x: np.ndarray, dims, inverse: bool = False) -> np.ndarray:
    """FP64 N-D arbiter (exact per-axis angle reduction), row-major."""
    return _nd(lib().orc_naive_dft_nd_f64, x, dims, inverse)


def naive_dft_nd_ref(x: np.ndarray, dims, inverse: bool = False) -> np.ndarray:
    """The reference's NaiveDFT2D/3D formula (internal/reference/dft2d.go,
    dft3d.go), complex128 result (the complex64 versions round it)."""
    return _nd(lib().orc_naive_dft_nd_ref, x, dims, inverse)


def algorithm(n: int) -> int:
    return lib().orc_algorithm(n)


def batch(x: np.ndarray, n: int, inverse: bool = False, nthreads: int = 1) -> np.ndarray:
    """Plan.ForwardBatch / InverseBatch restated; dtype picks c64/c128."""
    x = np.ascontiguousarray(x)
    count = x.size // n
    y = np.empty_like(x)
    if x.dtype == np.complex64:
        rc = lib().orc_batch_c64(_p(y), _p(x), n, count, int(inverse), nthreads)
    elif x.dtype == np.complex128:
        rc = lib().orc_batch_c128(_p(y), _p(x), n, count, int(inverse), nthreads)
    else:
        raise TypeError(x.dtype)
    if rc:
        raise RuntimeError(f"oracle batch failed rc={rc}")
    return y


def transform_algo(x: np.ndarray, algo: int, inverse: bool = False) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.complex64)
    y = np.empty_like(x)
    rc = lib().orc_transform_algo_c64(_p(y), _p(x), x.size, int(inverse), algo)
    if rc:
        raise RuntimeError(f"oracle transform rc={rc}")
    return y


def real_forward(x: np.ndarray, n: int, nthreads: int = 1) -> np.ndarray:
    x = np.ascontiguousarray(x)
    b = x.size // n
    if x.dtype == np.float32:
        y = np.empty(b * (n // 2 + 1), np.complex64)
        rc = lib().orc_real_forward_f32(_p(y), _p(x), n, b, nthreads)
    else:
        x = x.astype(np.float64)
        y = np.empty(b * (n // 2 + 1), np.complex128)
        rc = lib().orc_real_forward_f64(_p(y), _p(x), n, b)
    if rc:
        raise RuntimeError(f"oracle real forward rc={rc}")
    return y


def real_inverse(X: np.ndarray, n: int, nthreads: int = 1) -> np.ndarray:
    X = np.ascontiguousarray(X)
    b = X.size // (n // 2 + 1)
    if X.dtype == np.complex64:
        y = np.empty(b * n, np.float32)
        rc = lib().orc_real_inverse_f32(_p(y), _p(X), n, b, nthreads)
    else:
        X = X.astype(np.complex128)
        y = np.empty(b * n, np.float64)
        rc = lib().orc_real_inverse_f64(_p(y), _p(X), n, b)
    if rc:
        raise RuntimeError(f"oracle real inverse rc={rc}")
    return y


def convolve_real(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(b, dtype=np.float32)
    y = np.empty(a.size + b.size - 1, np.float32)
    rc = lib().orc_convolve_real_f32(_p(y), _p(a), a.size, _p(b), b.size)
    if rc:
        raise RuntimeError(f"oracle convolve_real rc={rc}")
    return y


def convolve(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.complex64)
    b = np.ascontiguousarray(b, dtype=np.complex64)
    y = np.empty(a.size + b.size - 1, np.complex64)
    rc = lib().orc_convolve_c64(_p(y), _p(a), a.size, _p(b), b.size)
    if rc:
        raise RuntimeError(f"oracle convolve rc={rc}")
    return y


def twiddles(n: int, c128: bool = False) -> np.ndarray:
    y = np.empty(n, np.complex128 if c128 else np.complex64)
    (lib().orc_twiddles_c128 if c128 else lib().orc_twiddles_c64)(_p(y), n)
    return y


def max_threads() -> int:
    return lib().orc_max_threads()
