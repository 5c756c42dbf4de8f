"""Parity of the sm_100a batched C2C path (Plan.ForwardBatch/InverseBatch)
with the CPU oracle, through the C ABI.  Tolerances: relative L2 error
<= 1e-6*log2N (complex64) and <= 1e-13*log2N (complex128) against FP64."""
import json
import os

import numpy as np
import pytest

import algofft
import oracle as O
from helpers import rel_l2, seeded_complex, tol_c2c

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))["cases"]


def _torch():
    import torch
    return torch


def _fp64_reference(x: np.ndarray, n: int, inverse=False) -> np.ndarray:
    """FP64 arbiter: the naive DFT for small n, else the oracle's complex128
    FFT (itself checked against the naive DFT on the CPU)."""
    x64 = x.astype(np.complex128)
    if n <= 512:
        return np.concatenate([O.naive_dft(x64[i:i + n], inverse) for i in range(0, x64.size, n)])
    return O.batch(x64, n, inverse=inverse)


def _run(plan, x: np.ndarray, count: int, inverse=False, inplace=False) -> np.ndarray:
    torch = _torch()
    src = torch.from_numpy(x).cuda()
    dst = src if inplace else torch.empty_like(src)
    if inverse:
        plan.InverseBatch(dst, src, count)
    else:
        plan.ForwardBatch(dst, src, count)
    torch.cuda.synchronize()
    return dst.cpu().numpy()


POW2_C64 = [2 ** k for k in range(1, 15)]
POW2_C128 = [2 ** k for k in range(1, 14)]


@pytest.mark.parametrize("n", POW2_C64)
def test_forward_batch_c64_pow2(n):
    count = max(3, min(64, (1 << 16) // n)) + 1  # ragged: not a multiple of the CTA batch
    x = seeded_complex(n * count, seed=n)
    with algofft.NewPlan(n) as p:
        y = _run(p, x, count)
    ref = _fp64_reference(x[: n * min(count, 8)], n)
    assert rel_l2(y[: ref.size], ref) <= tol_c2c(n, False)
    # every transform of the batch equals the CPU restatement of the reference path
    assert rel_l2(y, O.batch(x, n)) <= 2 * tol_c2c(n, False)


@pytest.mark.parametrize("n", POW2_C64)
def test_inverse_batch_c64_roundtrip(n):
    count = 5
    x = seeded_complex(n * count, seed=100 + n)
    with algofft.NewPlan(n) as p:
        X = _run(p, x, count)
        back = _run(p, X, count, inverse=True)
        ref_inv = _fp64_reference(X[: n * 2], n, inverse=True)
        y_inv = _run(p, X, count, inverse=True)
    assert rel_l2(y_inv[: ref_inv.size], ref_inv) <= tol_c2c(n, False)
    assert rel_l2(back, x) <= 2 * tol_c2c(n, False)


@pytest.mark.parametrize("n", POW2_C128)
def test_forward_inverse_c128_pow2(n):
    count = 7
    x = seeded_complex(n * count, seed=n, dtype=np.complex128)
    with algofft.NewPlan64(n) as p:
        y = _run(p, x, count)
        back = _run(p, y, count, inverse=True)
    ref = _fp64_reference(x, n)
    assert rel_l2(y, ref) <= tol_c2c(n, True)
    assert rel_l2(back, x) <= 2 * tol_c2c(n, True)


@pytest.mark.parametrize("n", [16, 1024, 16384])
def test_in_place_batch(n):
    count = 6
    x = seeded_complex(n * count, seed=9)
    with algofft.NewPlan(n) as p:
        a = _run(p, x, count)
        b = _run(p, x, count, inplace=True)
    assert np.array_equal(a, b)


def test_batch_equals_per_transform():
    # plan_batch_test.go:13-140: ForwardBatch equals a loop of Forward.
    n, count = 256, 10
    x = seeded_complex(n * count, seed=5)
    torch = _torch()
    with algofft.NewPlan(n) as p:
        batch = _run(p, x, count)
        singles = []
        for i in range(count):
            s = torch.from_numpy(x[i * n:(i + 1) * n].copy()).cuda()
            d = torch.empty_like(s)
            p.Forward(d, s)
            singles.append(d.cpu().numpy())
    assert np.array_equal(batch, np.concatenate(singles))


@pytest.mark.parametrize("case", [c for c in GOLDEN if c["kind"] in ("forward", "inverse")], ids=lambda c: c["name"])
def test_known_answers_on_gpu(case):
    dtype = np.complex128 if case["precision"] == "complex128" else np.complex64
    x = np.array([complex(a, b) for a, b in case["input"]], dtype=dtype)
    want = np.array([complex(a, b) for a, b in case["expected"]])
    n = case["n"]
    p = algofft.NewPlan64(n) if dtype == np.complex128 else algofft.NewPlan(n)
    with p:
        y = _run(p, x, 1, inverse=case["kind"] == "inverse")
    assert np.max(np.abs(y.astype(np.complex128) - want)) <= case["tol"]


@pytest.mark.parametrize("n", [65536, 16384, 1024])
def test_impulse_to_ones_c128(n):
    # precision_test.go:318-405: impulse -> all ones within 1e-11, round trip 1e-10.
    x = np.zeros(n, np.complex128)
    x[0] = 1
    with algofft.NewPlan64(n) as p:
        y = _run(p, x, 1)
        back = _run(p, y, 1, inverse=True)
    assert np.max(np.abs(y - 1)) <= 1e-11
    assert abs(back[0] - 1) <= 1e-10 and np.max(np.abs(back[1:])) <= 1e-10


def test_host_slices_match_device():
    n, count = 2048, 4
    x = seeded_complex(n * count, seed=21)
    with algofft.NewPlan(n) as p:
        dev = _run(p, x, count)
        host = np.empty_like(x)
        p.ForwardBatch(host, x, count)
    assert np.array_equal(dev, host)


def test_batch_argument_errors():
    # plan.go:504-516: nil -> ErrNilSlice, count < 1 -> ErrInvalidLength,
    # short slices -> ErrLengthMismatch.
    torch = _torch()
    n = 64
    with algofft.NewPlan(n) as p:
        a = torch.zeros(n * 4, dtype=torch.complex64, device="cuda")
        b = torch.zeros(n * 4, dtype=torch.complex64, device="cuda")
        with pytest.raises(algofft.ErrNilSlice):
            p.ForwardBatch(None, a, 1)
        with pytest.raises(algofft.ErrInvalidLength):
            p.ForwardBatch(a, b, 0)
        with pytest.raises(algofft.ErrLengthMismatch):
            p.ForwardBatch(a, b, 5)
        with pytest.raises(algofft.ErrLengthMismatch):
            p.Forward(a, b)  # single transform needs len == n exactly


@pytest.mark.parametrize("n,stride", [(1024, 4096), (64, 3), (16, 1)])
def test_strided_matches_contiguous(n, stride):
    # plan_strided_test.go:8-95: strided transform equals the contiguous one.
    torch = _torch()
    L = 1 + (n - 1) * stride
    x = seeded_complex(L, seed=31)
    with algofft.NewPlan(n) as p:
        src = torch.from_numpy(x).cuda()
        dst = torch.zeros_like(src)
        p.ForwardStrided(dst, src, stride)
        torch.cuda.synchronize()
        got = dst.cpu().numpy()[::stride][:n]
    ref = _fp64_reference(x[::stride][:n].copy(), n)
    assert rel_l2(got, ref) <= tol_c2c(n, False)
    with algofft.NewPlan(n) as p, pytest.raises(algofft.ErrInvalidStride):
        p.ForwardStrided(dst, src, 0)


# Two-pass (four-step, L2-resident) schedule for large N.
LARGE_C64 = [2 ** k for k in range(15, 25)]
LARGE_C128 = [2 ** k for k in range(14, 23)]


def _count_for(n, cap_elems=1 << 22):
    return max(1, min(5, cap_elems // n))


@pytest.mark.parametrize("n", LARGE_C64)
def test_forward_inverse_c64_large(n):
    count = _count_for(n)
    x = seeded_complex(n * count, seed=n % 9973)
    with algofft.NewPlan(n) as p:
        assert any(s in p.Algorithm() for s in ("-tp-", "-tp3-", "-tp3t-"))  # a multi-pass schedule
        y = _run(p, x, count)
        back = _run(p, y, count, inverse=True)
    ref = O.batch(x[: n * min(count, 2)].astype(np.complex128), n)
    assert rel_l2(y[: ref.size], ref) <= tol_c2c(n, False)
    assert rel_l2(back, x) <= 2 * tol_c2c(n, False)


@pytest.mark.parametrize("n", LARGE_C128)
def test_forward_inverse_c128_large(n):
    count = _count_for(n, 1 << 21)
    x = seeded_complex(n * count, seed=n % 9973, dtype=np.complex128)
    with algofft.NewPlan64(n) as p:
        y = _run(p, x, count)
        back = _run(p, y, count, inverse=True)
    ref = O.batch(x[: n * min(count, 2)], n)
    assert rel_l2(y[: ref.size], ref) <= tol_c2c(n, True)
    assert rel_l2(back, x) <= 2 * tol_c2c(n, True)


@pytest.mark.parametrize("n", [2 ** 15, 2 ** 20])
def test_large_in_place_and_many_groups(n):
    # enough transforms to cycle the scratch slots several times
    count = max(3, (1 << 24) // n) + 1
    x = seeded_complex(n * count, seed=77)
    with algofft.NewPlan(n) as p:
        a = _run(p, x, count)
        b = _run(p, x, count, inplace=True)
    assert np.array_equal(a, b)
    idx = [0, count // 2, count - 1]
    ref = O.batch(np.concatenate([x[i * n:(i + 1) * n] for i in idx]).astype(np.complex128), n)
    got = np.concatenate([a[i * n:(i + 1) * n] for i in idx])
    assert rel_l2(got, ref) <= tol_c2c(n, False)


@pytest.mark.parametrize("n", [4, 16, 32, 64, 128, 1024, 8192, 16384, 2 ** 15, 2 ** 16, 2 ** 17, 2 ** 20, 2 ** 22, 2 ** 24])
def test_every_variant_matches_oracle(n):
    count = max(2, (1 << 20) // n) + 3  # a partial last CTA for the batched kernels
    x = seeded_complex(n * count, seed=3 + n % 101)
    ref = O.batch(x[: 2 * n].astype(np.complex128), n)
    ref_tail = O.batch(x[-2 * n:].astype(np.complex128), n)
    toks = algofft.Variants(n)
    assert toks
    for tok in toks:
        with algofft.Plan(n, variant=tok) as p:
            assert p.Algorithm() == tok
            y = _run(p, x, count)
            back = _run(p, y, count, inverse=True)
            p.Check()
        assert rel_l2(y[: 2 * n], ref) <= tol_c2c(n, False), tok
        assert rel_l2(y[-2 * n:], ref_tail) <= tol_c2c(n, False), tok
        assert rel_l2(back, x) <= 2 * tol_c2c(n, False), tok


def test_autotune_feeds_plan_creation():
    algofft.ClearWisdom()
    try:
        rep = algofft.Autotune(4096, count=2048, iters=3)
        assert rep["best"] in algofft.Variants(4096)
        assert set(rep["variants"]) == set(algofft.Variants(4096))
        with algofft.NewPlan(4096) as p:
            assert p.Algorithm() == rep["best"]
        # PlannerMeasure tunes on first use of a length (measure.go:89-141)
        opts = algofft.PlanOptions(Planner=algofft.PlannerMeasure)
        with algofft.NewPlanWithOptions(2048, opts) as p:
            assert algofft.WisdomLen() == 2
            assert p.Algorithm() in algofft.Variants(2048)
    finally:
        algofft.ClearWisdom()


def test_forced_strategy_classes():
    n = 8192
    with algofft.NewPlanWithOptions(n, algofft.PlanOptions(Strategy=algofft.KernelSixStep)) as p:
        assert "-tp-" in p.Algorithm()
    with algofft.NewPlanWithOptions(n, algofft.PlanOptions(Strategy=algofft.KernelStockham)) as p:
        assert "-p2-" in p.Algorithm()



@pytest.mark.parametrize("n", [2 ** 21, 2 ** 24])
def test_three_pass_complex128(n):
    # the three-pass schedule (N = N1 x M1 x M2, factors <= 256) in complex128
    tok = [t for t in algofft.Variants(n, algofft.COMPLEX128) if "-tp3-" in t]
    assert tok
    x = seeded_complex(2 * n, seed=n % 89, dtype=np.complex128)
    with algofft.Plan(n, algofft.COMPLEX128, variant=tok[0]) as p:
        y = _run(p, x, 2)
        back = _run(p, y, 2, inverse=True)
    assert rel_l2(y[:n], np.fft.fft(x[:n])) <= tol_c2c(n, True)
    assert rel_l2(back, x) <= 2 * tol_c2c(n, True)



@pytest.mark.parametrize("n,prec", [(2 ** 21, algofft.COMPLEX64), (2 ** 23, algofft.COMPLEX64),
                                    (2 ** 21, algofft.COMPLEX128), (2 ** 24, algofft.COMPLEX128)])
def test_tma_three_pass_variants(n, prec):
    # the TMA-staged three-pass kernels (persistent, tiles copied by the copy
    # engine) give the FP64 results within the stated tolerance
    c128 = prec == algofft.COMPLEX128
    toks = [t for t in algofft.Variants(n, prec) if "-tp3t-" in t]
    assert len(toks) >= 2
    count = 3
    x = seeded_complex(count * n, seed=n % 83, dtype=np.complex128 if c128 else np.complex64)
    ref = np.fft.fft(x[:n].astype(np.complex128))
    for tok in toks:
        with algofft.Plan(n, prec, variant=tok) as p:
            assert p.Algorithm() == tok
            y = _run(p, x, count)
            back = _run(p, y, count, inverse=True)
            p.Check()
        assert rel_l2(y[:n], ref) <= tol_c2c(n, c128), tok
        assert rel_l2(back, x) <= 2 * tol_c2c(n, c128), tok


def test_tma_three_pass_unaligned_buffers():
    # a source and destination 8 bytes off a 16-byte boundary cannot be
    # addressed by the copy engine: the plan takes the plain kernels
    import torch
    n, count = 2 ** 21, 2
    tok = [t for t in algofft.Variants(n) if "-tp3t-" in t][0]
    x = seeded_complex(count * n, seed=9)
    raw = torch.zeros(count * n + 1, dtype=torch.complex64, device="cuda")
    raw[1:] = torch.from_numpy(x).cuda()
    out = torch.zeros_like(raw)
    src, dst = raw[1:], out[1:]
    assert src.data_ptr() % 16 == 8
    with algofft.Plan(n, variant=tok) as p:
        p.ForwardBatch(dst, src, count)
        torch.cuda.synchronize()
        p.Check()
    y = dst.cpu().numpy()
    assert rel_l2(y[:n], np.fft.fft(x[:n].astype(np.complex128))) <= tol_c2c(n, False)
    assert rel_l2(y[n:], np.fft.fft(x[n:].astype(np.complex128))) <= tol_c2c(n, False)
