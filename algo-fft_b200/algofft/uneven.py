"""Uneven-length batches (thousands of transforms of different lengths)."""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import check, lib
from .plan import COMPLEX64, PlanOptions, _ptr_len, _stream


class PlanUneven:
    """Transforms of the given lengths packed back to back."""

    def __init__(self, lengths, precision: int = COMPLEX64, opts: PlanOptions | None = None):
        self.lengths = np.ascontiguousarray(np.asarray(lengths, dtype=np.int64))
        self.offsets = np.concatenate([[0], np.cumsum(self.lengths)[:-1]]).astype(np.int64)
        self._h = ctypes.c_void_p()
        c = (opts or PlanOptions()).to_c()
        arr = self.lengths.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        check(lib().gfft_plan_uneven_new(ctypes.byref(self._h), precision, self.lengths.size, arr, ctypes.byref(c)))

    def Close(self):
        if self._h:
            lib().gfft_plan_uneven_close(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.Close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.Close()

    def Total(self) -> int:
        return int(lib().gfft_plan_uneven_total(self._h))

    def Forward(self, dst, src, graph: bool = True):
        dp, _, _ = _ptr_len(dst)
        sp, _, _ = _ptr_len(src)
        check(lib().gfft_uneven_exec(self._h, -1, dp, sp, int(graph), _stream(dst)))

    def Inverse(self, dst, src, graph: bool = True):
        dp, _, _ = _ptr_len(dst)
        sp, _, _ = _ptr_len(src)
        check(lib().gfft_uneven_exec(self._h, 1, dp, sp, int(graph), _stream(dst)))

    def ForwardPerSize(self, dst, src):
        dp, _, _ = _ptr_len(dst)
        sp, _, _ = _ptr_len(src)
        check(lib().gfft_uneven_exec_per_size(self._h, -1, dp, sp, _stream(dst)))


def _primes(lo: int, hi: int) -> np.ndarray:
    sieve = np.ones(hi + 1, dtype=bool)
    sieve[:2] = False
    for i in range(2, int(hi ** 0.5) + 1):
        if sieve[i]:
            sieve[i * i::i] = False
    p = np.nonzero(sieve)[0]
    return p[(p >= lo) & (p <= hi)]


def _smooth7(hi: int) -> np.ndarray:
    out = []
    a = 1
    while a <= hi:
        b = a
        while b <= hi:
            c = b
            while c <= hi:
                d = c
                while d <= hi:
                    out.append(d)
                    d *= 7
                c *= 5
            b *= 3
        a *= 2
    v = np.array(sorted(out), dtype=np.int64)
    return v[(v & (v - 1)) != 0]  # not powers of two


def uneven_lengths(count: int = 20000, seed: int = 0) -> np.ndarray:
    """The uneven workload: 50% powers of two 2^6..2^16, 30% 7-smooth lengths
    <= 65536 that are not powers of two, 20% primes in [1009, 65521]."""
    rng = np.random.default_rng(seed)
    kind = rng.random(count)
    pow2 = 2 ** rng.integers(6, 17, count)
    sm = _smooth7(65536)
    pr = _primes(1009, 65521)
    smooth = sm[rng.integers(0, sm.size, count)]
    prime = pr[rng.integers(0, pr.size, count)]
    return np.where(kind < 0.5, pow2, np.where(kind < 0.8, smooth, prime)).astype(np.int64)
