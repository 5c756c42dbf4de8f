"""Accuracy of the four-step twiddle of the runtime two-pass pass 1, restated
in numpy float32: W_N^(n2 k1) taken from the two-level table (W^(hi 2^s) *
W^(lo)) every fourth column n2 and, between, stepped by one product with
W_N^(k1).  Checked over every (n2, k1) pair of N = 50421 = 147 x 343 and a
sample of N = 10^6 against the exact value: the stepped twiddles stay within
a few units in the last place of the gathered ones."""
import numpy as np


def _tables(n):
    shift = 0
    while (1 << (2 * shift)) < n:
        shift += 1
    nlo = 1 << shift
    nhi = (n + nlo - 1) >> shift
    lo = np.exp(-2j * np.pi * np.arange(nlo) / n).astype(np.complex64)
    hi = np.exp(-2j * np.pi * (np.arange(nhi) * nlo) / n).astype(np.complex64)
    return lo, hi, shift, nlo - 1


def _cmul(a, b):
    """float32 complex product as the device forms it (four products, two sums)."""
    ar, ai = a.real.astype(np.float32), a.imag.astype(np.float32)
    br, bi = b.real.astype(np.float32), b.imag.astype(np.float32)
    return (ar * br - ai * bi).astype(np.float32) + 1j * (ar * bi + ai * br).astype(np.float32)


def _stepped(n, n1, n2_cols, k1):
    lo, hi, shift, mask = _tables(n)
    step = _cmul(hi[k1 >> shift], lo[k1 & mask])
    out = np.empty((len(n2_cols), len(k1)), np.complex128)
    w = None
    for c, n2 in enumerate(n2_cols):
        if c % 4 == 0:
            m = n2 * k1
            w = _cmul(hi[m >> shift], lo[m & mask])
        else:
            w = _cmul(w, step)
        out[c] = w
    return out


def _gathered(n, n2_cols, k1):
    lo, hi, shift, mask = _tables(n)
    m = np.asarray(n2_cols)[:, None] * k1[None, :]
    return _cmul(hi[m >> shift], lo[m & mask])


def _exact(n, n2_cols, k1):
    m = (np.asarray(n2_cols, dtype=np.int64)[:, None] * k1[None, :]) % n
    return np.exp(-2j * np.pi * m / n)


def _check(n, n1, n2):
    k1 = np.arange(n1, dtype=np.int64)
    worst_s = worst_g = 0.0
    for col0 in range(0, n2, 16):             # the CTA tiles of 16 columns
        cols = list(range(col0, min(col0 + 16, n2)))
        ex = _exact(n, cols, k1)
        worst_s = max(worst_s, float(np.abs(_stepped(n, n1, cols, k1) - ex).max()))
        worst_g = max(worst_g, float(np.abs(_gathered(n, cols, k1) - ex).max()))
    return worst_s, worst_g


def test_stepped_twiddle_error_n50421():
    s, g = _check(50421, 147, 343)
    ulp = 2.0 ** -24
    assert g <= 4 * ulp
    assert s <= 8 * ulp, (s / ulp, g / ulp)   # measured 4.7 ulp (gather alone 1.9)


def test_stepped_twiddle_error_n1e6_sample():
    n, n1, n2 = 1000000, 1000, 1000
    k1 = np.arange(n1, dtype=np.int64)
    ulp = 2.0 ** -24
    for col0 in (0, 496, 992 - 16 * 3):
        cols = list(range(col0, col0 + 16))
        err = float(np.abs(_stepped(n, n1, cols, k1) - _exact(n, cols, k1)).max())
        assert err <= 8 * ulp, err / ulp
