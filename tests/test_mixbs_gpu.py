"""Bluestein on FFT lengths that are not powers of two: the chain of
gfft_mixbs.cuh (chirp-weighted loads, filter-product stores, inverse first
pass, chirp stores) over M = M1 x M2 >= 2n - 1, M1 and M2 compiled column
lengths (multiples of 16 up to 512), used when M is below NextPow2(2n - 1),
the reference's choice (plan.go:865, plan_bluestein.go:7-58).  Results
against numpy's FP64 FFT, forward and inverse, both precisions, batched and
at a batch distance larger than the length."""
import numpy as np
import pytest

import algofft
from helpers import rel_l2, seeded_complex, tol_c2c

pytestmark = pytest.mark.gpu

SB = [L for L in range(48, 513, 16) if all(L % p for p in (11, 13, 17, 19, 23, 29, 31))]


def _smooth7(n):
    for p in (2, 3, 5, 7):
        while n % p == 0:
            n //= p
    return n == 1


def _lengths(n):
    """(mixed FFT length or 0, NextPow2(2n - 1)): the smallest product of two
    compiled lengths >= 2n - 1 where it is below the power of two (beyond
    the one-CTA range)."""
    lens = [L for L in SB if _smooth7(L)]
    best = min(a * b for i, a in enumerate(lens) for b in lens[i:] if a * b >= 2 * n - 1)
    p2 = 1 << (2 * n - 2).bit_length()
    return (best if best < p2 and p2 > 16384 else 0), p2


def _mixed_m(n):
    mx, p2 = _lengths(n)
    return mx or p2


def _preferred(mx, p2):
    """The automatic choice's rule (bs_mixed_preferred, gfft_plans.cu): the
    mixed length up to the power of two itself for 32768, 0.9 of it for
    65536, 0.70 beyond."""
    r = 1.0 if p2 <= 32768 else 0.9 if p2 <= 65536 else 0.70
    return mx > 0 and mx <= r * p2


def _plan(n, prec=0):
    """The mixed chain where it exists (forced: the automatic choice
    weighs it against the power of two), else the default plan."""
    mx, _ = _lengths(n)
    tok = f"gpu-sm100-bluestein-n{n}-mx" if mx else None
    return algofft.Plan(n, prec, variant=tok)


def _run(p, x, count, inverse=False):
    import torch
    src = torch.from_numpy(x).cuda()
    dst = torch.empty_like(src)
    (p.InverseBatch if inverse else p.ForwardBatch)(dst, src, count)
    torch.cuda.synchronize()
    p.Check()
    return dst.cpu().numpy()


# primes from just past the one-CTA limit (8209: M = 17920 for 32768) to
# 100003 (200704 for 262144), a composite with a large prime factor, two
# lengths whose best product is the power of two itself, and lengths on
# either side of the rule (28753: 0.88 of 65536, 31657: 0.98, 42043: 0.66
# of 131072, 45737: 0.70)
C64 = [8209, 12289, 16411, 20011, 40009, 49233, 100003, 65521, 131071, 28753, 31657, 42043, 45737]


@pytest.mark.parametrize("n", C64)
def test_default_bluestein_length(n):
    """The automatic choice: the mixed length where the rule prefers it
    ("-mx"), else the power of two ("-p2" where a smaller mixed length was
    passed over)."""
    mx, p2 = _lengths(n)
    with algofft.NewPlan(n) as p:
        alg = p.Algorithm()
    if _preferred(mx, p2):
        assert alg.startswith(f"gpu-sm100-bluestein-n{n}-mx-m{mx}+"), alg
    elif mx:
        assert alg.startswith(f"gpu-sm100-bluestein-n{n}-p2-m{p2}+"), alg
    else:
        assert alg.startswith(f"gpu-sm100-bluestein-n{n}-m{p2}+"), alg
    toks = [t for t in algofft.Variants(n) if "bluestein" in t]
    assert toks == ([f"gpu-sm100-bluestein-n{n}-mx", f"gpu-sm100-bluestein-n{n}-p2"] if mx else [])


@pytest.mark.parametrize("n", C64)
def test_mixed_bluestein_c64(n):
    M = _mixed_m(n)
    count = max(2, min(4, (1 << 21) // n))
    x = seeded_complex(n * count, seed=n % 1000)
    with _plan(n) as p:
        alg = p.Algorithm()
        assert f"-m{M}+" in alg, alg
        y = _run(p, x, count)
        back = _run(p, y, count, inverse=True)
    ref = np.fft.fft(x.astype(np.complex128).reshape(count, n), axis=1).ravel()
    assert rel_l2(y, ref) <= 2 * tol_c2c(M, False)
    assert rel_l2(back, x) <= 4 * tol_c2c(M, False)


@pytest.mark.parametrize("n", [8209, 16411, 40009, 100003])
def test_mixed_bluestein_c128(n):
    M = _mixed_m(n)
    count = 2
    x = seeded_complex(n * count, seed=n % 1000, dtype=np.complex128)
    with _plan(n, algofft.COMPLEX128) as p:
        assert f"-m{M}+" in p.Algorithm()
        y = _run(p, x, count)
        back = _run(p, y, count, inverse=True)
    ref = np.fft.fft(x.reshape(count, n), axis=1).ravel()
    assert rel_l2(y, ref) <= 2 * tol_c2c(M, True)
    assert rel_l2(back, x) <= 4 * tol_c2c(M, True)


def test_mixed_bluestein_batch_distance():
    """Transforms dist > n apart (gfft_exec_strided_batch at stride 1): the
    chain reads and writes each transform at its own offset and leaves the
    gaps alone."""
    import torch
    n, count, dist = 16411, 3, 16411 + 37
    x = seeded_complex(dist * count, seed=9)
    with _plan(n) as p:
        src = torch.from_numpy(x).cuda()
        dst = torch.zeros_like(src)
        p.StridedBatch(dst, src, count, 1, dist)
        torch.cuda.synchronize()
        got = dst.cpu().numpy()
    M = _mixed_m(n)
    for b in range(count):
        ref = np.fft.fft(x[b * dist:b * dist + n].astype(np.complex128))
        assert rel_l2(got[b * dist:b * dist + n], ref) <= 2 * tol_c2c(M, False)
        assert not np.any(got[b * dist + n:(b + 1) * dist])
