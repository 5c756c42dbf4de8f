"""Host-side selection of the compiled mixed-radix variants, through the C
ABI without a GPU (gfft_plan_variants): which lengths get a compiled single
pass, which four-step split the compiled column tiles take, and which
Bluestein lengths get a mixed FFT length, against a restatement of the
rules in Python."""
import pytest

import algofft


def _smooth7(n):
    for p in (2, 3, 5, 7):
        while n % p == 0:
            n //= p
    return n == 1


TABLE = [L for L in range(48, 1025) if _smooth7(L)]
BS = [80] + [L for L in range(112, 513) if _smooth7(L) and L % 16 == 0]


def _mix_split(n):
    """Largest table length d <= sqrt(n) with n / d in the table (0: none)."""
    best = 0
    for d in TABLE:
        if n % d == 0 and d * d <= n and (n // d) in TABLE:
            best = max(best, d)
    return best


def _rows(n, prec):
    top = 12288 if prec == 0 else 6144
    return n in TABLE or (1024 < n <= top and _smooth7(n) and n & (n - 1))


def _bs_mixed(n):
    """Smallest product of two Bluestein factor lengths >= 2n - 1 when below
    NextPow2(2n - 1) and beyond the one-CTA range (0: none)."""
    p2 = 1 << (2 * n - 2).bit_length()
    m = min(a * b for i, a in enumerate(BS) for b in BS[i:] if a * b >= 2 * n - 1) if 2 * n - 1 <= 512 * 512 else 0
    return m if p2 > 16384 and 0 < m < p2 else 0


SMOOTH = [60, 100, 343, 1000, 1080, 6000, 6561, 10000, 12000, 13440, 21609, 50421, 100000, 117649, 250000,
          1000000, 1008000, 7 ** 7, 2 * 3 ** 12]


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("n", SMOOTH)
def test_compiled_mixed_radix_variants(n, prec):
    v = algofft.Variants(n, prec)
    assert (f"gpu-sm100-mixr-n{n}" in v) == bool(_rows(n, prec))
    d = _mix_split(n)
    mixc = [t for t in v if "-mixc-" in t]
    assert mixc == ([f"gpu-sm100-mixc-{d}x{n // d}"] if d else []), (n, v)


@pytest.mark.parametrize("n", [8191, 8209, 12289, 16411, 20011, 40009, 65521, 100003, 131071, 262147])
def test_bluestein_length_variants(n):
    v = [t for t in algofft.Variants(n) if "bluestein" in t]
    mx = _bs_mixed(n)
    assert v == ([f"gpu-sm100-bluestein-n{n}-mx", f"gpu-sm100-bluestein-n{n}-p2"] if mx else []), (n, v)
