"""Parity of the non-power-of-two paths: runtime-radix Stockham for 7-smooth
lengths (mixedradix.go) and Bluestein for the rest (plan_bluestein.go)."""
import numpy as np
import pytest

import algofft
import oracle as O
from helpers import rel_l2, seeded_complex, tol_c2c

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def _run(plan, x, count, inverse=False, inplace=False):
    torch = _torch()
    src = torch.from_numpy(x).cuda()
    dst = src if inplace else torch.empty_like(src)
    (plan.InverseBatch if inverse else plan.ForwardBatch)(dst, src, count)
    torch.cuda.synchronize()
    plan.Check()
    return dst.cpu().numpy()


def _judge(x, n, inverse=False):
    x64 = x.astype(np.complex128)
    if n <= 2048:
        return np.concatenate([O.naive_dft(x64[i:i + n], inverse) for i in range(0, x64.size, n)])
    return np.concatenate([np.fft.ifft(x64[i:i + n]) if inverse else np.fft.fft(x64[i:i + n])
                           for i in range(0, x64.size, n)])


# 2/3/5-smooth (the reference's mixed radix), 7-smooth (radix 7), and the
# runtime two-pass range (> one CTA).
SMOOTH = [3, 5, 6, 7, 9, 12, 15, 21, 49, 60, 100, 243, 343, 360, 1000, 2187, 3125, 6000, 6720, 15625,
          2 * 3 * 5 * 7 * 64, 48000, 50421, 62500, 65536 + 0 * 1]
PRIMES = [2, 11, 13, 17, 31, 97, 251, 1009, 4099, 8191, 16411, 65521, 131071, 262147]


@pytest.mark.parametrize("n", SMOOTH)
def test_mixed_radix_c64(n):
    count = max(2, min(9, (1 << 20) // n))
    x = seeded_complex(n * count, seed=n)
    with algofft.NewPlan(n) as p:
        y = _run(p, x, count)
        back = _run(p, y, count, inverse=True)
    k = min(count, 3)
    assert rel_l2(y[: k * n], _judge(x[: k * n], n)) <= tol_c2c(n, False)
    assert rel_l2(back, x) <= 2 * tol_c2c(n, False)


@pytest.mark.parametrize("n", [3, 9, 12, 81, 343, 2187, 6000, 50421])
def test_mixed_radix_c128(n):
    count = 3
    x = seeded_complex(n * count, seed=n, dtype=np.complex128)
    with algofft.NewPlan64(n) as p:
        y = _run(p, x, count)
        back = _run(p, y, count, inverse=True)
    assert rel_l2(y, _judge(x, n)) <= tol_c2c(n, True)
    assert rel_l2(back, x) <= 2 * tol_c2c(n, True)


@pytest.mark.parametrize("n", PRIMES)
def test_bluestein_c64(n):
    count = max(2, min(6, (1 << 19) // n))
    x = seeded_complex(n * count, seed=n)
    with algofft.NewPlan(n) as p:
        assert n <= 7 or "bluestein" in p.Algorithm() or "p2" in p.Algorithm()
        y = _run(p, x, count)
        back = _run(p, y, count, inverse=True)
    assert rel_l2(y[: 2 * n], _judge(x[: 2 * n], n)) <= tol_c2c(n, False)
    assert rel_l2(back, x) <= 2 * tol_c2c(n, False)


@pytest.mark.parametrize("n", [7, 31, 1021, 16411, 65521, 131071])
def test_bluestein_c128(n):
    # exact k^2 mod 2n chirps keep complex128 Bluestein at 1e-13*log2N even
    # where the reference's float64(k*k) chirp (bluestein.go:23-29) cannot
    count = 2
    x = seeded_complex(n * count, seed=n, dtype=np.complex128)
    with algofft.NewPlanWithOptions(n, algofft.PlanOptions(Strategy=algofft.KernelBluestein),
                                    precision=algofft.COMPLEX128) as p:
        assert "bluestein" in p.Algorithm()
        y = _run(p, x, count)
        back = _run(p, y, count, inverse=True)
    assert rel_l2(y, _judge(x, n)) <= tol_c2c(n, True)
    assert rel_l2(back, x) <= 2 * tol_c2c(n, True)


@pytest.mark.parametrize("n", [7, 13, 29, 31])
def test_bluestein_matches_reference_primes(n):
    # plan_bluestein_test.go:243-330 sizes; also the oracle's restatement of
    # the reference Bluestein path agrees within the reference's 1e-3.
    x = seeded_complex(n, seed=1)
    with algofft.NewPlan(n) as p:
        y = _run(p, x, 1)
    assert np.max(np.abs(y - O.batch(x, n))) <= 1e-3
    assert rel_l2(y, _judge(x, n)) <= tol_c2c(n, False)


def test_forced_bluestein_on_pow2_and_smooth():
    for n in (1024, 360):
        x = seeded_complex(4 * n, seed=2)
        opts = algofft.PlanOptions(Strategy=algofft.KernelBluestein)
        with algofft.NewPlanWithOptions(n, opts) as p:
            assert "bluestein" in p.Algorithm()
            y = _run(p, x, 4)
        assert rel_l2(y, _judge(x, n)) <= tol_c2c(n, False)


@pytest.mark.parametrize("n", [360, 4099])
def test_non_pow2_in_place(n):
    x = seeded_complex(3 * n, seed=4)
    with algofft.NewPlan(n) as p:
        a = _run(p, x, 3)
        b = _run(p, x, 3, inplace=True)
    assert np.array_equal(a, b)
