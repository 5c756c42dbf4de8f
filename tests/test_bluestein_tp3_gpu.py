"""Bluestein on FFT lengths M = 2^21..2^24 (primes n = 2^19 + 21 .. 2^22 +
15): the chain fused into the plain three-pass FFT_M (kernels_bluestein_tp3.cu:
chirp-weighted zero-padded loads in the forward first pass, the filter
product in the forward third pass's stores, chirp, 1/M and 1/n in the
inverse third pass's stores of the n outputs), the reference's
NextPow2(2n - 1) padding (plan.go:865, plan_bluestein.go:7-58).  Results
against numpy's FP64 FFT, forward and inverse, both precisions, and at a
batch distance larger than the length."""
import numpy as np
import pytest

import algofft
from helpers import rel_l2, seeded_complex, tol_c2c

pytestmark = pytest.mark.gpu

# (prime n, M = NextPow2(2n - 1))
CASES = [(524309, 1 << 21), (1048583, 1 << 22), (2097169, 1 << 23), (4194319, 1 << 24)]


def _run(p, x, count, inverse=False):
    import torch
    src = torch.from_numpy(x).cuda()
    dst = torch.empty_like(src)
    (p.InverseBatch if inverse else p.ForwardBatch)(dst, src, count)
    torch.cuda.synchronize()
    p.Check()
    return dst.cpu().numpy()


@pytest.mark.parametrize("n,M", CASES)
def test_three_pass_chain_c64(n, M):
    count = 2
    x = seeded_complex(n * count, seed=n % 1000)
    with algofft.NewPlan(n) as p:
        alg = p.Algorithm()
        assert alg.startswith(f"gpu-sm100-bluestein-n{n}-m{M}+gpu-sm100-tp3-"), alg
        y = _run(p, x, count)
        back = _run(p, y, count, inverse=True)
    ref = np.fft.fft(x.astype(np.complex128).reshape(count, n), axis=1).ravel()
    assert rel_l2(y, ref) <= 2 * tol_c2c(M, False)
    assert rel_l2(back, x) <= 4 * tol_c2c(M, False)


@pytest.mark.parametrize("n,M", [CASES[0], CASES[2]])
def test_three_pass_chain_c128(n, M):
    x = seeded_complex(n, seed=n % 1000, dtype=np.complex128)
    with algofft.Plan(n, algofft.COMPLEX128) as p:
        assert f"-m{M}+gpu-sm100-tp3-" in p.Algorithm()
        y = _run(p, x, 1)
        back = _run(p, y, 1, inverse=True)
    ref = np.fft.fft(x)
    assert rel_l2(y, ref) <= 2 * tol_c2c(M, True)
    assert rel_l2(back, x) <= 4 * tol_c2c(M, True)


def test_three_pass_chain_batch_distance_and_in_place():
    """Transforms dist > n apart: each read and written at its own offset,
    the gaps left alone; in place equal to out of place."""
    import torch
    n, count, dist = 524309, 3, 524309 + 29
    x = seeded_complex(dist * count, seed=17)
    with algofft.NewPlan(n) as p:
        src = torch.from_numpy(x).cuda()
        dst = torch.zeros_like(src)
        p.StridedBatch(dst, src, count, 1, dist)
        same = src.clone()
        p.StridedBatch(same, same, count, 1, dist)
        torch.cuda.synchronize()
        got, inplace = dst.cpu().numpy(), same.cpu().numpy()
    for b in range(count):
        seg = slice(b * dist, b * dist + n)
        ref = np.fft.fft(x[seg].astype(np.complex128))
        assert rel_l2(got[seg], ref) <= 2 * tol_c2c(1 << 21, False)
        assert not np.any(got[b * dist + n:(b + 1) * dist])
    np.testing.assert_array_equal(inplace[:n], got[:n])
