"""Tensor-core precision form (split fp16 hi+lo operands, FP32 accumulation
on tcgen05.mma) against the FP64 FFT: the stated complex64 tolerance,
rel L2 <= 1e-6 * log2 N, on both input sets of the precision comparison
(i.i.d. N(0,1), and log-uniform magnitudes 1e-4..1e4 with uniform phase).
Powers of two that are not powers of 16 (n = r * 16^s, r = 2, 4, 8) run a
leading FP32 radix-r stage before the radix-16 tensor-core stages."""
import numpy as np
import pytest

import algofft
from helpers import rel_l2, tol_c2c

pytestmark = pytest.mark.gpu


def _inputs(kind, total, seed):
    rng = np.random.default_rng(seed)
    if kind == "normal":
        return (rng.standard_normal(total) + 1j * rng.standard_normal(total)).astype(np.complex64)
    mag = 10 ** rng.uniform(-4, 4, total)
    return (mag * np.exp(1j * rng.uniform(0, 2 * np.pi, total))).astype(np.complex64)


def _tc(n):
    return algofft.Plan(n, algofft.COMPLEX64, variant=f"gpu-sm100-tc16-n{n}")


@pytest.mark.parametrize("n", [16, 32, 64, 256, 512, 2048, 4096, 8192, 65536, 1 << 17, 1 << 20, 1 << 21,
                               1 << 22, 1 << 23, 1 << 24])
@pytest.mark.parametrize("kind", ["normal", "loguniform"])
def test_tc_forward_inverse(n, kind):
    import torch
    count = max(1, (1 << 20) // n)
    x = _inputs(kind, n * count, seed=n)
    with _tc(n) as p:
        assert p.Algorithm() == f"gpu-sm100-tc16-n{n}"
        src = torch.from_numpy(x).cuda()
        y = torch.empty_like(src)
        p.ForwardBatch(y, src, count)
        back = torch.empty_like(src)
        p.InverseBatch(back, y, count)
        torch.cuda.synchronize()
        p.Check()
        yh, bh = y.cpu().numpy(), back.cpu().numpy()
    k = min(count, 4)
    ref = np.fft.fft(x[:k * n].reshape(k, n).astype(np.complex128), axis=1).ravel()
    assert rel_l2(yh[:k * n], ref) <= tol_c2c(n, False)
    assert np.max(np.abs(yh[:k * n] - ref)) <= 4 * tol_c2c(n, False) * np.max(np.abs(ref))
    assert rel_l2(bh, x) <= 2 * tol_c2c(n, False)


@pytest.mark.parametrize("n,count", [(16, 100), (32, 77), (256, 3), (4096, 1), (8192, 3), (65536, 1),
                                     (1 << 21, 1)])
def test_tc_ragged_batch_and_in_place(n, count):
    import torch
    x = _inputs("normal", n * count, seed=count)
    with _tc(n) as p:
        t = torch.from_numpy(x).cuda()
        ref_dev = torch.empty_like(t)
        p.ForwardBatch(ref_dev, t, count)
        p.ForwardBatch(t, t, count)  # in place
        torch.cuda.synchronize()
        got = t.cpu().numpy()
    assert np.array_equal(got, ref_dev.cpu().numpy())
    ref = np.fft.fft(x.reshape(count, n).astype(np.complex128), axis=1).ravel()
    assert rel_l2(got, ref) <= tol_c2c(n, False)


def test_tc_rejects_other_lengths():
    for n in (2, 8, 12288, 1000, 1 << 25):
        with pytest.raises(algofft.ErrNotImplemented):
            _tc(n)
