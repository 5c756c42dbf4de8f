"""Parity of the N-D plans (Plan2D/3D/ND, PlanReal2D/3D) and batched strided
transforms with numpy's FP64 FFTs, through the C ABI."""
import math

import numpy as np
import pytest

import algofft
from helpers import rel_l2, seeded_complex, tol_c2c

pytestmark = pytest.mark.gpu


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


def _tol(dims, c128=False):
    return tol_c2c(int(np.prod(dims)), c128) * 1.5


@pytest.mark.parametrize("dims", [(8, 8), (16, 32), (64, 48), (17, 31), (3, 1024), (1024, 3), (1, 64), (2048, 512)])
def test_plan2d_c64(dims):
    import torch
    x = seeded_complex(int(np.prod(dims)), seed=sum(dims))
    with algofft.NewPlan2D(*dims) as p:
        src = _dev(x)
        dst = torch.empty_like(src)
        p.Forward(dst, src)
        back = torch.empty_like(src)
        p.Inverse(back, dst)
        y, b = _host(dst), _host(back)
    ref = np.fft.fft2(x.reshape(dims).astype(np.complex128)).ravel()
    assert rel_l2(y, ref) <= _tol(dims)
    assert rel_l2(b, x) <= 2 * _tol(dims)


@pytest.mark.parametrize("dims", [(8, 16, 32), (5, 6, 7), (4, 6, 8, 10), (32, 32, 32)])
def test_plan_nd_c64_and_in_place(dims):
    x = seeded_complex(int(np.prod(dims)), seed=7)
    with algofft.NewPlanND(dims) as p:
        t = _dev(x)
        p.ForwardInPlace(t)
        y = _host(t)
    assert rel_l2(y, np.fft.fftn(x.reshape(dims).astype(np.complex128)).ravel()) <= _tol(dims)


@pytest.mark.parametrize("dims", [(16, 16), (24, 40), (7, 11, 13)])
def test_plan_nd_c128(dims):
    x = seeded_complex(int(np.prod(dims)), seed=5, dtype=np.complex128)
    with algofft.PlanND(dims, algofft.COMPLEX128) as p:
        y = np.empty_like(x)
        p.Forward(y, x)
        b = np.empty_like(x)
        p.Inverse(b, y)
    assert rel_l2(y, np.fft.fftn(x.reshape(dims)).ravel()) <= _tol(dims, True)
    assert rel_l2(b, x) <= 2 * _tol(dims, True)


def test_plan2d_batch_stride():
    rows, cols, batch, stride = 8, 16, 3, 200
    x = seeded_complex(batch * stride, seed=11)
    opts = algofft.PlanOptions(Batch=batch, Stride=stride)
    with algofft.NewPlan2D(rows, cols, opts=opts) as p:
        y = np.zeros_like(x)
        p.Forward(y, x)
    for b in range(batch):
        seg = x[b * stride:b * stride + rows * cols].reshape(rows, cols).astype(np.complex128)
        assert rel_l2(y[b * stride:b * stride + rows * cols], np.fft.fft2(seg).ravel()) <= _tol((rows, cols))
    with pytest.raises(algofft.ErrInvalidStride):
        algofft.NewPlan2D(rows, cols, opts=algofft.PlanOptions(Batch=2, Stride=10)).Forward(y, x)


def test_plan2d_config_shape_4096():
    # the 2-D complex64 4096 x 4096 exercise shape (batch reduced to 2)
    import torch
    dims, batch = (4096, 4096), 2
    g = torch.Generator(device="cuda")
    g.manual_seed(0)
    x = torch.randn(2 * batch * dims[0] * dims[1], generator=g, device="cuda").view(torch.complex64)
    with algofft.NewPlan2D(*dims, opts=algofft.PlanOptions(Batch=batch)) as p:
        y = torch.empty_like(x)
        p.Forward(y, x)
        back = torch.empty_like(x)
        p.Inverse(back, y)
        torch.cuda.synchronize()
    err = (torch.linalg.vector_norm(back - x) / torch.linalg.vector_norm(x)).item()
    assert err <= 2 * _tol(dims)
    ref = torch.fft.fft2(x[: dims[0] * dims[1]].view(dims).to(torch.complex128))
    got = y[: dims[0] * dims[1]].view(dims).to(torch.complex128)
    assert (torch.linalg.vector_norm(got - ref) / torch.linalg.vector_norm(ref)).item() <= _tol(dims)


@pytest.mark.parametrize("dims", [(16, 32), (64, 100), (6, 10, 12), (256, 256, 256)])
def test_plan_real_nd(dims):
    import torch
    n = int(np.prod(dims))
    x = np.random.default_rng(3).uniform(-1, 1, n).astype(np.float32)
    p = algofft.NewPlanReal2D(*dims) if len(dims) == 2 else algofft.NewPlanReal3D(*dims)
    with p:
        assert p.SpectrumLen() == n // dims[-1] * (dims[-1] // 2 + 1)
        src = _dev(x)
        X = torch.empty(p.SpectrumLen(), dtype=torch.complex64, device="cuda")
        p.Forward(X, src)
        back = torch.empty_like(src)
        p.Inverse(back, X)
        full = torch.empty(n, dtype=torch.complex64, device="cuda")
        p.ForwardFull(full, src)
        back2 = torch.empty_like(src)
        p.InverseFull(back2, full)
        Xh, bh, fh, b2 = _host(X), _host(back), _host(full), _host(back2)
    x64 = x.reshape(dims).astype(np.float64)
    assert rel_l2(Xh, np.fft.rfftn(x64).ravel()) <= _tol(dims)
    assert rel_l2(fh, np.fft.fftn(x64).ravel()) <= _tol(dims)
    assert rel_l2(bh, x) <= 2 * _tol(dims)
    assert rel_l2(b2, x) <= 2 * _tol(dims)


def test_strided_column_batch_config_shape():
    # 4096 columns of length 1024 at stride 4096 (the strided exercise shape)
    import torch
    n, cols = 1024, 4096
    x = seeded_complex(n * cols, seed=13)
    with algofft.NewPlan(n) as p:
        src = _dev(x)
        dst = torch.empty_like(src)
        p.StridedBatch(dst, src, count=cols, stride=cols, dist=1)
        y = _host(dst)
    ref = np.fft.fft(x.reshape(n, cols).astype(np.complex128), axis=0).ravel()
    assert rel_l2(y, ref) <= tol_c2c(n, False)


@pytest.mark.parametrize("n,count,stride,dist", [(64, 5, 3, 400), (1009, 4, 2, 2500), (360, 7, 9, 1)])
def test_strided_batch_general(n, count, stride, dist):
    import torch
    L = (count - 1) * dist + (n - 1) * stride + 1
    x = seeded_complex(L, seed=n)
    with algofft.NewPlan(n) as p:
        src = _dev(x)
        dst = torch.zeros_like(src)
        p.StridedBatch(dst, src, count=count, stride=stride, dist=dist)
        y = _host(dst)
    for b in range(count):
        idx = b * dist + np.arange(n) * stride
        assert rel_l2(y[idx], np.fft.fft(x[idx].astype(np.complex128))) <= tol_c2c(n, False)


def test_nd_errors():
    with pytest.raises(algofft.ErrInvalidLength):
        algofft.NewPlanND((4, 0))
    with pytest.raises(algofft.ErrInvalidLength):
        algofft.NewPlanReal2D(4, 7)
    with algofft.NewPlan2D(4, 4) as p:
        with pytest.raises(algofft.ErrLengthMismatch):
            p.Forward(np.zeros(15, np.complex64), np.zeros(16, np.complex64))


# ---- the reference's N-D oracle cases (fixtures) -----------------------------
import json  # noqa: E402
import os  # noqa: E402

ND_CASES = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "nd_known_answers.json")))["cases"]


def _fixture_c(v, c128):
    a = np.asarray(v, dtype=np.float64)
    return (a[..., 0] + 1j * a[..., 1]).astype(np.complex128 if c128 else np.complex64)


@pytest.mark.parametrize("case", ND_CASES, ids=lambda c: c["name"])
def test_nd_plans_match_reference_oracle_cases(case):
    """Plan2D / Plan3D against the cases of plan_2d_test.go:202-383 and
    plan_3d_test.go:237-380: every element within the reference test's own
    absolute tolerance of the exact DFT, and the whole within the stated
    relative L2 bound."""
    import torch
    c128 = case["precision"] == "complex128"
    prec = algofft.COMPLEX128 if c128 else algofft.COMPLEX64
    dims = tuple(case["dims"])
    n = int(np.prod(dims))
    tol = tol_c2c(n, c128)
    if case["kind"] == "forward_batch":
        batch, stride = case["batch"], case["stride"]
        src = np.zeros(batch * stride, np.complex64)
        for b, sig in enumerate(case["input"]):
            src[b * stride:b * stride + n] = _fixture_c(sig, False)
        with algofft.PlanND(dims, prec, opts=algofft.PlanOptions(Batch=batch, Stride=stride)) as p:
            d_src = _dev(src)
            d_dst = torch.zeros_like(d_src)
            p.Forward(d_dst, d_src)
            y = _host(d_dst)
        for b, want in enumerate(case["expected"]):
            w = _fixture_c(want, True).astype(np.complex128)
            got = y[b * stride:b * stride + n]
            assert np.max(np.abs(got - w)) <= case["tol_abs"]
            assert rel_l2(got, w) <= tol
        return
    x = _fixture_c(case["input"], c128)
    want = _fixture_c(case["expected"], True).astype(np.complex128)
    with algofft.PlanND(dims, prec) as p:
        d_src = _dev(x)
        d_dst = torch.empty_like(d_src)
        (p.Inverse if case["kind"] == "inverse" else p.Forward)(d_dst, d_src)
        y = _host(d_dst)
    assert np.max(np.abs(y - want)) <= case["tol_abs"]
    assert rel_l2(y, want) <= tol
