"""Convolve / Correlate / ConvolveReal (convolve.go, convolve_real.go,
correlate.go) over the C ABI.  numpy arrays run the host path, torch CUDA
tensors the device path."""
from __future__ import annotations

from ._lib import ErrNilSlice, check, lib
from .plan import COMPLEX64, COMPLEX128, _ptr_len, _stream


def _prec(x, real: bool) -> int:
    s = str(x.dtype)
    if real:
        return COMPLEX128 if s.endswith("float64") else COMPLEX64
    return COMPLEX128 if s.endswith("complex128") else COMPLEX64


def _call(dev, host, real, dst, a, b):
    if dst is None or a is None or b is None:
        raise ErrNilSlice("algo-fft: nil slice")
    dp, dl, dd = _ptr_len(dst)
    ap, al, _ = _ptr_len(a)
    bp, bl, _ = _ptr_len(b)
    prec = _prec(a, real)
    if dd:
        check(getattr(lib(), dev)(prec, dp, dl, ap, al, bp, bl, _stream(dst)))
    else:
        check(getattr(lib(), host)(prec, dp, dl, ap, al, bp, bl))


def Convolve(dst, a, b):
    """convolve.go:9 (complex64) / :65 Convolve128 (complex128)."""
    _call("gfft_convolve", "gfft_convolve_host", False, dst, a, b)


Convolve128 = Convolve


def CrossCorrelate(dst, a, b):
    """correlate.go:13 (Correlate is the same call)."""
    _call("gfft_correlate", "gfft_correlate_host", False, dst, a, b)


Correlate = CrossCorrelate
Correlate128 = CrossCorrelate
CrossCorrelate128 = CrossCorrelate


def AutoCorrelate(dst, a):
    """correlate.go:38."""
    CrossCorrelate(dst, a, a)


AutoCorrelate128 = AutoCorrelate


def ConvolveReal(dst, a, b):
    """convolve_real.go:9 (float32; float64 inputs use double precision)."""
    _call("gfft_convolve_real", "gfft_convolve_real_host", True, dst, a, b)


def ConvolveRealBatch(dst, a, a_len: int, count: int, b, a_dist: int | None = None, dst_dist: int | None = None):
    """count signals of a_len reals (device tensors) convolved with one kernel b."""
    a_dist = a_len if a_dist is None else a_dist
    dst_dist = a_len + b.numel() - 1 if dst_dist is None else dst_dist
    dp, _, _ = _ptr_len(dst)
    ap, _, _ = _ptr_len(a)
    bp, bl, _ = _ptr_len(b)
    check(lib().gfft_convolve_real_batch(_prec(a, True), dp, dst_dist, ap, a_len, a_dist, count, bp, bl, _stream(dst)))
