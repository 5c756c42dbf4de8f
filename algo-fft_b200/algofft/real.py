"""Real-input plans: PlanRealT[F, C] (plan_real_generic.go) over the C ABI."""
from __future__ import annotations

import ctypes

from ._lib import ErrNilSlice, check, lib
from .plan import COMPLEX64, COMPLEX128, PlanOptions, _ptr_len, _stream


class PlanReal:
    """NewPlanReal32 (precision COMPLEX64: float32/complex64) or NewPlanReal64."""

    def __init__(self, n: int, precision: int = COMPLEX64, opts: PlanOptions | None = None):
        self._h = ctypes.c_void_p()
        self.precision = precision
        c = (opts or PlanOptions()).to_c()
        check(lib().gfft_plan_real_new(ctypes.byref(self._h), precision, n, ctypes.byref(c)))

    def Close(self):
        if self._h:
            lib().gfft_plan_real_close(self._h)
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

    def Len(self) -> int:
        return int(lib().gfft_plan_real_len(self._h))

    def SpectrumLen(self) -> int:
        return int(lib().gfft_plan_real_spectrum_len(self._h))

    def _fwd(self, dst, src, scaling):
        if dst is None or src is None:
            raise ErrNilSlice("algo-fft: nil slice")
        dp, dl, dd = _ptr_len(dst)
        sp, sl, sd = _ptr_len(src)
        if dd:
            check(lib().gfft_real_forward(self._h, scaling, dp, dl, sp, sl, _stream(dst)))
        else:
            check(lib().gfft_real_forward_host(self._h, scaling, dp, dl, sp, sl))

    def Forward(self, dst, src):
        """plan_real_generic.go:111 (dst: n/2+1 bins, src: n reals)."""
        self._fwd(dst, src, 0)

    def ForwardNormalized(self, dst, src):
        """plan_real_generic.go:231 (x 1/n)."""
        self._fwd(dst, src, 1)

    def ForwardUnitary(self, dst, src):
        """plan_real_generic.go:243 (x 1/sqrt(n))."""
        self._fwd(dst, src, 2)

    def Inverse(self, dst, src):
        """plan_real_generic.go:256 (dst: n reals, src: n/2+1 bins)."""
        if dst is None or src is None:
            raise ErrNilSlice("algo-fft: nil slice")
        dp, dl, dd = _ptr_len(dst)
        sp, sl, sd = _ptr_len(src)
        if dd:
            check(lib().gfft_real_inverse(self._h, dp, dl, sp, sl, _stream(dst)))
        else:
            check(lib().gfft_real_inverse_host(self._h, dp, dl, sp, sl))


def NewPlanReal(n: int) -> PlanReal:
    """plan_real.go NewPlanReal (float32)."""
    return PlanReal(n, COMPLEX64)


def NewPlanReal32(n: int) -> PlanReal:
    """plan_real_constructors.go:8."""
    return PlanReal(n, COMPLEX64)


def NewPlanReal64(n: int) -> PlanReal:
    """plan_real_constructors.go:20."""
    return PlanReal(n, COMPLEX128)


def NewPlanRealWithOptions(n: int, opts: PlanOptions, precision: int = COMPLEX64) -> PlanReal:
    return PlanReal(n, precision, opts)
