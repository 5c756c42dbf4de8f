"""Every compiled mixed-radix kernel against numpy's FP64 FFT: the single
pass (rows mode) of every 7-smooth length it is built for, both precisions;
every column length as both passes of the four-step of L x L; and every
Bluestein factor length in each role it can take (M1: the chirp-weighted
first pass and the output pass; M2: the fused middle pass) through primes
whose mixed FFT length M = M1 x M2 uses it there.  The
reference runs these lengths through its mixed-radix recursion and
Bluestein (internal/fft/mixedradix.go:45-188, plan_bluestein.go:7-58)."""
import numpy as np
import pytest

import algofft
from helpers import rel_l2, seeded_complex, tol_c2c

pytestmark = pytest.mark.gpu


def _smooth7(n):
    for p in (2, 3, 5, 7):
        while n % p == 0:
            n //= p
    return n == 1


TABLE = [L for L in range(48, 1025) if _smooth7(L)]
ROWS3 = {0: [L for L in range(1025, 12289) if _smooth7(L) and L & (L - 1)],
         1: [L for L in range(1025, 6145) if _smooth7(L) and L & (L - 1)]}
# primes whose mixed Bluestein lengths M = M1 x M2 (M1 <= M2) take every
# factor length as M1 and as M2 where some n in 8193..131072 does (512 is
# never M1, 80, 112 and 128 never M2)
BS_PRIMES = [8209, 8963, 9221, 10369, 12289, 15361, 17921, 18433, 19207, 20483, 25097, 28687, 30727, 40961, 48397,
             49157, 72577, 76801, 80021, 80651, 92173, 98317, 114689]


def _check(tok, n, prec, count, bound):
    import torch
    dt = np.complex128 if prec else np.complex64
    x = seeded_complex(n * count, seed=n % 997, dtype=dt)
    with algofft.Plan(n, prec, variant=tok) as p:
        assert p.Algorithm().startswith(tok), (p.Algorithm(), tok)
        src = torch.from_numpy(x).cuda()
        dst = torch.empty_like(src)
        p.ForwardBatch(dst, src, count)
        torch.cuda.synchronize()
        p.Check()
        y = dst.cpu().numpy()
    ref = np.fft.fft(x.astype(np.complex128).reshape(count, n), axis=1).ravel()
    err = rel_l2(y, ref)
    assert err <= bound, (tok, err, bound)


@pytest.mark.parametrize("prec", [0, 1])
def test_every_single_pass_length(prec):
    for n in TABLE + ROWS3[prec]:
        _check(f"gpu-sm100-mixr-n{n}", n, prec, 3, tol_c2c(n, bool(prec)))


@pytest.mark.parametrize("prec", [0, 1])
def test_every_column_length_in_both_passes(prec):
    for L in TABLE:
        n = L * L
        _check(f"gpu-sm100-mixc-{L}x{L}", n, prec, 1, tol_c2c(n, bool(prec)))


@pytest.mark.parametrize("prec", [0, 1])
def test_every_bluestein_factor_length(prec):
    for n in BS_PRIMES:
        m = 1 << (2 * n - 2).bit_length()
        _check(f"gpu-sm100-bluestein-n{n}-mx", n, prec, 2, 2 * tol_c2c(m, bool(prec)))
