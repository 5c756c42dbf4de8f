"""Parity of the real-input path (PlanReal Forward/Inverse,
plan_real_generic.go) with the oracle and the FP64 arbiter."""
import json
import os

import numpy as np
import pytest

import algofft
import oracle as O
from helpers import rel_l2, tol_c2c

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))["cases"]


def _reals(count, seed, dtype=np.float32):
    return np.random.default_rng(seed).uniform(-1, 1, count).astype(dtype)


@pytest.mark.parametrize("case", [c for c in GOLDEN if c["kind"] == "r2c"], ids=lambda c: c["name"])
def test_real_known_answers(case):
    x = np.array(case["input"], np.float32)
    want = np.array([complex(a, b) for a, b in case["expected"]])
    with algofft.NewPlanReal(case["n"]) as p:
        got = np.empty(p.SpectrumLen(), np.complex64)
        p.Forward(got, x)
    assert np.max(np.abs(got - want)) <= case["tol"]


# h = n/2: fused single-pass (pow2 <= 16384), two-pass (32768), 7-smooth
# (3000, 5), Bluestein (1009), and the trivial n = 2.
SIZES = [2, 4, 10, 16, 32, 1024, 4096, 8192, 32768, 65536, 6000, 2018]


@pytest.mark.parametrize("n", SIZES)
def test_real_forward_inverse_c64(n):
    import torch
    batch = max(2, min(16, (1 << 20) // n))
    x = _reals(n * batch, seed=n)
    opts = algofft.PlanOptions(Batch=batch)
    with algofft.NewPlanRealWithOptions(n, opts) as p:
        h1 = p.SpectrumLen()
        src = torch.from_numpy(x).cuda()
        X = torch.empty(batch * h1, dtype=torch.complex64, device="cuda")
        p.Forward(X, src)
        back = torch.empty_like(src)
        p.Inverse(back, X)
        torch.cuda.synchronize()
        Xh = X.cpu().numpy()
        back = back.cpu().numpy()
    ref = np.fft.rfft(x.reshape(batch, n).astype(np.float64), axis=1).ravel()
    assert rel_l2(Xh, ref) <= tol_c2c(n, False)
    assert rel_l2(Xh[: 2 * h1], O.real_forward(x[: 2 * n], n)) <= 2 * tol_c2c(n, False)
    assert rel_l2(back, x) <= 2 * tol_c2c(n, False)


@pytest.mark.parametrize("n", [16, 4096, 65536, 6000])
def test_real_forward_inverse_c128(n):
    x = _reals(n * 3, seed=n, dtype=np.float64)
    with algofft.PlanReal(n, algofft.COMPLEX128, algofft.PlanOptions(Batch=3)) as p:
        X = np.empty(3 * p.SpectrumLen(), np.complex128)
        p.Forward(X, x)
        back = np.empty_like(x)
        p.Inverse(back, X)
    ref = np.fft.rfft(x.reshape(3, n), axis=1).ravel()
    assert rel_l2(X, ref) <= tol_c2c(n, True)
    assert rel_l2(back, x) <= 2 * tol_c2c(n, True)


def test_real_batch_stride_layout():
    # plan_real_test.go:38-88: Batch with Stride applies to reals and bins.
    n, batch, stride = 64, 5, 70
    x = _reals(batch * stride, seed=3)
    opts = algofft.PlanOptions(Batch=batch, Stride=stride)
    with algofft.NewPlanRealWithOptions(n, opts) as p:
        X = np.zeros(batch * stride, np.complex64)
        p.Forward(X, x)
        back = np.zeros_like(x)
        p.Inverse(back, X)
    for b in range(batch):
        ref = np.fft.rfft(x[b * stride:b * stride + n].astype(np.float64))
        assert rel_l2(X[b * stride:b * stride + n // 2 + 1], ref) <= tol_c2c(n, False)
        assert rel_l2(back[b * stride:b * stride + n], x[b * stride:b * stride + n]) <= 2 * tol_c2c(n, False)
    with pytest.raises(algofft.ErrInvalidStride):
        algofft.NewPlanRealWithOptions(n, algofft.PlanOptions(Batch=2, Stride=n - 1)).Forward(X, x)


def test_real_scaling_variants():
    n = 1024
    x = _reals(n, seed=9)
    ref = np.fft.rfft(x.astype(np.float64))
    with algofft.NewPlanReal(n) as p:
        for fn, s in ((p.Forward, 1.0), (p.ForwardNormalized, 1.0 / n), (p.ForwardUnitary, n ** -0.5)):
            X = np.empty(n // 2 + 1, np.complex64)
            fn(X, x)
            assert rel_l2(X, ref * s) <= tol_c2c(n, False)


def test_real_errors():
    with pytest.raises(algofft.ErrInvalidLength):
        algofft.NewPlanReal(7)
    with algofft.NewPlanReal(16) as p:
        x = np.zeros(16, np.float32)
        with pytest.raises(algofft.ErrLengthMismatch):
            p.Forward(np.zeros(8, np.complex64), x)
        X = np.zeros(9, np.complex64)
        X[0] = 1 + 1j  # DC must be real (plan_real_generic.go:301-316)
        with pytest.raises(algofft.ErrInvalidSpectrum):
            p.Inverse(x, X)
        X[0] = 1
        X[8] = 2 + 0.5j
        with pytest.raises(algofft.ErrInvalidSpectrum):
            p.Inverse(x, X)


def test_real_full_size_r2c_roundtrip():
    # the R2C config: N = 4096, batch 65536 (1 GiB of float32 input)
    import torch
    n, batch = 4096, 65536
    g = torch.Generator(device="cuda")
    g.manual_seed(0)
    x = torch.rand(n * batch, generator=g, device="cuda") * 2 - 1
    with algofft.NewPlanRealWithOptions(n, algofft.PlanOptions(Batch=batch)) as p:
        X = torch.empty(batch * (n // 2 + 1), dtype=torch.complex64, device="cuda")
        p.Forward(X, x)
        back = torch.empty_like(x)
        p.Inverse(back, X)
        torch.cuda.synchronize()
    err = (torch.linalg.vector_norm(back - x) / torch.linalg.vector_norm(x)).item()
    assert err <= 2 * tol_c2c(n, False)
    idx = [0, batch // 2, batch - 1]
    xs = x.view(batch, n)[idx].cpu().numpy().astype(np.float64)
    Xs = X.view(batch, n // 2 + 1)[idx].cpu().numpy()
    assert rel_l2(Xs, np.fft.rfft(xs, axis=1)) <= tol_c2c(n, False)
