"""N-D plans: Plan2D/Plan3D/PlanND and PlanReal2D/PlanReal3D over the C ABI."""
from __future__ import annotations

import ctypes

from ._lib import ErrNilSlice, check, lib
from .plan import COMPLEX64, COMPLEX128, PlanOptions, _ptr_len, _stream


class PlanND:
    def __init__(self, dims, precision: int = COMPLEX64, real: bool = False, opts: PlanOptions | None = None):
        self._h = ctypes.c_void_p()
        self.dims = tuple(int(d) for d in dims)
        self.precision = precision
        arr = (ctypes.c_int64 * max(1, len(self.dims)))(*self.dims)
        c = (opts or PlanOptions()).to_c()
        check(lib().gfft_plan_nd_new(ctypes.byref(self._h), precision, len(self.dims), arr, int(real),
                                     ctypes.byref(c)))

    def Close(self):
        if self._h:
            lib().gfft_plan_nd_close(self._h)
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
        return int(lib().gfft_plan_nd_len(self._h))

    def SpectrumLen(self) -> int:
        return int(lib().gfft_plan_nd_spectrum_len(self._h))

    def _call(self, dev, host, dst, src):
        if dst is None or src is None:
            raise ErrNilSlice("algo-fft: nil slice")
        dp, dl, dd = _ptr_len(dst)
        sp, sl, sd = _ptr_len(src)
        if dd:
            check(getattr(lib(), dev)(self._h, dp, dl, sp, sl, _stream(dst)))
        elif host is None:
            raise TypeError("this call takes device buffers")
        else:
            check(getattr(lib(), host)(self._h, dp, dl, sp, sl))

    def Forward(self, dst, src):
        self._call("gfft_nd_forward", "gfft_nd_forward_host", dst, src)

    def Inverse(self, dst, src):
        self._call("gfft_nd_inverse", "gfft_nd_inverse_host", dst, src)

    def ForwardInPlace(self, data):
        self.Forward(data, data)

    def InverseInPlace(self, data):
        self.Inverse(data, data)

    def ForwardFull(self, dst, src):
        """plan_real_2d.go:231 (device buffers)."""
        self._call("gfft_nd_forward_full", None, dst, src)

    def InverseFull(self, dst, src):
        """plan_real_2d.go:370 (device buffers)."""
        self._call("gfft_nd_inverse_full", None, dst, src)


def NewPlan2D(rows: int, cols: int, precision: int = COMPLEX64, opts: PlanOptions | None = None) -> PlanND:
    """plan_2d.go:28 NewPlan2D[T]."""
    return PlanND((rows, cols), precision, False, opts)


def NewPlan3D(depth: int, height: int, width: int, precision: int = COMPLEX64,
              opts: PlanOptions | None = None) -> PlanND:
    """plan_3d.go:42 NewPlan3D[T]."""
    return PlanND((depth, height, width), precision, False, opts)


def NewPlanND(dims, precision: int = COMPLEX64, opts: PlanOptions | None = None) -> PlanND:
    """plan_nd.go:43 NewPlanND[T]."""
    return PlanND(dims, precision, False, opts)


def NewPlanReal2D(rows: int, cols: int, opts: PlanOptions | None = None, precision: int = COMPLEX64) -> PlanND:
    """plan_real_2d.go:43 NewPlanReal2D."""
    return PlanND((rows, cols), precision, True, opts)


def NewPlanReal3D(depth: int, height: int, width: int, opts: PlanOptions | None = None,
                  precision: int = COMPLEX64) -> PlanND:
    """plan_real_3d.go:42 NewPlanReal3D."""
    return PlanND((depth, height, width), precision, True, opts)
