"""Property tests of the GPU path, the families of the reference's own suite
(precision_test.go:13-316, internal/fft/properties_test.go,
plan_fuzz_test.go:9-140, concurrent_test.go:12-400): Parseval, linearity,
the shift theorem, complex64 against complex128, error accumulation over
many round trips, bit-exact determinism, concurrent use of one plan, and a
seeded fuzz over lengths -- across every schedule class (single pass,
two-pass, three-pass, runtime radix, Bluestein, uneven batch)."""
import threading

import numpy as np
import pytest
from hypothesis import given, settings, strategies as st

import algofft
from helpers import rel_l2, seeded_complex, tol_c2c

pytestmark = pytest.mark.gpu

# one length per schedule class: single pass, two-pass, three-pass,
# runtime radix, runtime two-pass, Bluestein (small and large M)
CLASSES = [1024, 1 << 16, 1 << 21, 6000, 50421, 1009, 65521]


def _fwd(plan, x, count, inverse=False):
    import torch
    src = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    dst = torch.empty_like(src)
    (plan.InverseBatch if inverse else plan.ForwardBatch)(dst, src, count)
    torch.cuda.synchronize()
    return dst.cpu().numpy()


@pytest.mark.parametrize("n", CLASSES)
def test_parseval_linearity_shift(n):
    count = 2
    x = seeded_complex(n * count, seed=n % 101)
    y = seeded_complex(n * count, seed=n % 103 + 1)
    with algofft.NewPlan(n) as p:
        X, Y = _fwd(p, x, count), _fwd(p, y, count)
        a, b = np.complex64(0.75 - 0.5j), np.complex64(-1.25 + 0.25j)
        L = _fwd(p, (a * x + b * y).astype(np.complex64), count)
        s = 7 % n
        Xs = _fwd(p, np.concatenate([np.roll(x[i * n:(i + 1) * n], s) for i in range(count)]), count)
    tol = tol_c2c(4 * n, False)
    # Parseval: sum |X|^2 = n sum |x|^2
    ex = np.sum(np.abs(x.astype(np.complex128)) ** 2)
    eX = np.sum(np.abs(X.astype(np.complex128)) ** 2) / n
    assert abs(eX - ex) <= 4 * tol * ex
    # linearity: F(a x + b y) = a F(x) + b F(y)
    assert rel_l2(L, a.astype(np.complex128) * X + b.astype(np.complex128) * Y) <= 2 * tol
    # shift: F(x[(j - s) mod n])[k] = F(x)[k] W_n^{k s}
    k = np.arange(n)
    w = np.exp(-2j * np.pi * k * s / n)
    want = np.concatenate([X[i * n:(i + 1) * n].astype(np.complex128) * w for i in range(count)])
    assert rel_l2(Xs, want) <= 2 * tol


@pytest.mark.parametrize("n", [64, 4096, 65536, 1009, 6000])
def test_complex64_agrees_with_complex128(n):
    # precision_test.go:196-316: max relative difference <= 1e-5
    x = seeded_complex(n, seed=n % 97, dtype=np.complex128)
    with algofft.NewPlan(n) as p32, algofft.NewPlan64(n) as p64:
        a = _fwd(p32, x.astype(np.complex64), 1).astype(np.complex128)
        b = _fwd(p64, x, 1)
    assert np.max(np.abs(a - b)) <= 1e-5 * np.max(np.abs(b))


@pytest.mark.parametrize("n", [1024, 1 << 16, 1 << 21, 1009])
def test_error_accumulation_over_round_trips(n):
    # precision_test.go:13-91: 100 forward + inverse cycles stay within a
    # bound that grows no faster than the cycle count
    import torch
    x = seeded_complex(n, seed=5)
    with algofft.NewPlan(n) as p:
        t = torch.from_numpy(x).cuda()
        for _ in range(100):
            p.ForwardBatch(t, t, 1)
            p.InverseBatch(t, t, 1)
        torch.cuda.synchronize()
        back = t.cpu().numpy()
    assert rel_l2(back, x) <= 100 * 2 * tol_c2c(n, False)


@pytest.mark.parametrize("n", CLASSES)
def test_determinism(n):
    # plan_fuzz_test.go: the same input gives the same output, bit for bit
    x = seeded_complex(3 * n, seed=11)
    with algofft.NewPlan(n) as p:
        a = _fwd(p, x, 3)
        b = _fwd(p, x, 3)
    assert np.array_equal(a, b)


def test_uneven_determinism():
    import torch
    L = algofft.uneven_lengths(300, seed=4)
    with algofft.PlanUneven(L) as p:
        x = torch.from_numpy(seeded_complex(p.Total(), seed=2)).cuda()
        y1, y2 = torch.empty_like(x), torch.empty_like(x)
        p.Forward(y1, x)
        p.Forward(y2, x)
        torch.cuda.synchronize()
    assert torch.equal(y1, y2)


@pytest.mark.parametrize("n", [4096, 1 << 17, 6000, 1009])
def test_one_plan_from_many_threads(n):
    # concurrent_test.go:12-400: a plan shared by threads, each on its own
    # stream, gives the sequential results
    import torch
    count, threads = 4, 6
    xs = [seeded_complex(n * count, seed=100 + i) for i in range(threads)]
    with algofft.NewPlan(n) as p:
        want = [_fwd(p, x, count) for x in xs]
        outs = [None] * threads
        errs = []

        def work(i):
            try:
                s = torch.cuda.Stream()
                with torch.cuda.stream(s):
                    src = torch.from_numpy(xs[i]).cuda()
                    dst = torch.empty_like(src)
                    for _ in range(3):
                        p.ForwardBatch(dst, src, count)
                    s.synchronize()
                    outs[i] = dst.cpu().numpy()
            except Exception as e:  # surfaced below
                errs.append(e)

        ts = [threading.Thread(target=work, args=(i,)) for i in range(threads)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
    assert not errs
    for i in range(threads):
        assert np.array_equal(outs[i], want[i])


@settings(max_examples=40, deadline=None, derandomize=True)
@given(n=st.integers(min_value=1, max_value=70000), count=st.integers(min_value=1, max_value=3))
def test_fuzz_round_trip(n, count):
    # plan_fuzz_test.go:9-140: any length plans, runs and round-trips
    x = seeded_complex(n * count, seed=n % 1009)
    with algofft.NewPlan(n) as p:
        y = _fwd(p, x, count)
        back = _fwd(p, y, count, inverse=True)
    m = 1
    while m < 2 * n:
        m <<= 1
    tol = tol_c2c(max(m, 2), False)
    assert np.all(np.isfinite(y))
    assert rel_l2(back, x) <= 4 * tol
    ref = np.fft.fft(x[:n].astype(np.complex128))
    assert rel_l2(y[:n], ref) <= 2 * tol
