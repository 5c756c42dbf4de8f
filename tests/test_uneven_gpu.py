"""Parity of uneven-length batches (many transforms of different lengths
packed back to back) with numpy's FP64 FFT per transform, through the C ABI.
The reference runs such a workload as a loop of Plan.Forward over one plan
per length; gfft_uneven_exec_per_size is that loop on the GPU, and the
batched path must agree with it."""
import numpy as np
import pytest

import algofft
from helpers import rel_l2, seeded_complex, tol_c2c

pytestmark = pytest.mark.gpu

# every route of the plan: 1 and 2, CTA-sized 7-smooth, CTA-sized Bluestein
# (primes), large powers of two (gathered per length), large 7-smooth (the
# mixed-radix four-step, one launch per factor length: 13440 = 112 x 120,
# 21609 = 147 x 147 and 50421 = 147 x 343 share a pass-1 launch, 25000 =
# 125 x 200 and 40000 = 200 x 200 a pass-2 launch), large primes (Bluestein
# items on mixed FFT lengths where the plans' rule prefers them: 16411 twice
# at 144 x 240, 12289, 20011, 40009; grouped by power-of-two FFT length
# otherwise: 31657, 65521), repeats of one length
LENGTHS = [1, 2, 3, 5, 7, 8, 13, 64, 97, 360, 1009, 1024, 2048, 4099, 5003, 6000, 8191, 12289, 16384,
           25000, 32768, 40000, 65521, 65536, 1009, 64, 65536, 360, 131072, 1 << 20, 13440, 21609, 50421,
           50421, 62500, 40000, 16411, 20011, 40009, 16411, 31657]


def _tol(n, c128):
    if n & (n - 1):  # Bluestein runs two FFTs of length NextPow2(2n-1)
        m = 1
        while m < 2 * n - 1:
            m <<= 1
        return 2 * tol_c2c(m, c128)
    return tol_c2c(n, c128)


def _check(lengths, y, x, inverse, c128):
    off = 0
    for n in lengths:
        seg = x[off:off + n].astype(np.complex128)
        want = np.fft.ifft(seg) if inverse else np.fft.fft(seg)
        assert rel_l2(y[off:off + n], want) <= _tol(n, c128), (n, rel_l2(y[off:off + n], want))
        off += n


@pytest.mark.parametrize("c128", [False, True])
def test_uneven_parity(c128):
    import torch
    prec = algofft.COMPLEX128 if c128 else algofft.COMPLEX64
    dt = np.complex128 if c128 else np.complex64
    with algofft.PlanUneven(LENGTHS, prec) as p:
        total = p.Total()
        assert total == sum(LENGTHS)
        x = seeded_complex(total, seed=3, dtype=dt)
        src = torch.from_numpy(x).cuda()
        y = torch.empty_like(src)
        p.Forward(y, src)
        back = torch.empty_like(src)
        p.Inverse(back, y)
        torch.cuda.synchronize()
        yh, bh = y.cpu().numpy(), back.cpu().numpy()
    _check(LENGTHS, yh, x, False, c128)
    _check(LENGTHS, bh, yh, True, c128)


def test_uneven_graph_direct_per_size_and_in_place():
    import torch
    L = [7, 4099, 64, 32768, 24000, 3, 65521, 1024, 5003, 100]
    with algofft.PlanUneven(L) as p:
        x = seeded_complex(p.Total(), seed=8)
        src = torch.from_numpy(x).cuda()
        outs = []
        for graph in (True, True, False):  # capture, replay, direct launches
            y = torch.empty_like(src)
            p.Forward(y, src, graph=graph)
            outs.append(y)
        ps = torch.empty_like(src)
        p.ForwardPerSize(ps, src)
        ip = src.clone()
        p.Forward(ip, ip)
        torch.cuda.synchronize()
    a = outs[0].cpu().numpy()
    assert np.array_equal(a, outs[1].cpu().numpy())
    assert np.array_equal(a, outs[2].cpu().numpy())
    assert np.array_equal(a, ip.cpu().numpy())
    _check(L, ps.cpu().numpy(), x, False, False)
    _check(L, a, x, False, False)


def test_uneven_workload_sample():
    # a 600-transform sample of the uneven workload's length mix
    import torch
    L = algofft.uneven_lengths(600, seed=1)
    with algofft.PlanUneven(L) as p:
        x = seeded_complex(p.Total(), seed=2)
        src = torch.from_numpy(x).cuda()
        y = torch.empty_like(src)
        p.Forward(y, src)
        torch.cuda.synchronize()
        yh = y.cpu().numpy()
    # every one of the 600 transforms against numpy's FP64 FFT
    _check(L, yh, x, False, False)


def test_uneven_errors():
    with pytest.raises(algofft.ErrInvalidLength):
        algofft.PlanUneven([4, 0, 8])
    with pytest.raises(algofft.ErrInvalidLength):
        algofft.PlanUneven([(1 << 24) + 1])


def test_uneven_calls_on_two_streams_at_once():
    """Two threads, each on its own stream, call one plan at the same time
    (graph replay and direct launches, more distinct buffers than the plan
    keeps graphs for): every transform of every call matches numpy's FP64
    FFT (the calls share the plan's work buffers and must not overlap)."""
    import threading
    import torch
    L = [64, 4099, 32768, 24000, 65521, 1024, 5003, 100, 131072]
    with algofft.PlanUneven(L) as p:
        total = p.Total()
        xs = [seeded_complex(total, seed=30 + i) for i in range(2)]
        srcs = [torch.from_numpy(x).cuda() for x in xs]
        outs = [[torch.empty_like(srcs[i]) for _ in range(6)] for i in range(2)]
        torch.cuda.synchronize()
        errors = []

        def worker(i):
            try:
                s = torch.cuda.Stream()
                with torch.cuda.stream(s):
                    for rep in range(3):
                        for j, y in enumerate(outs[i]):
                            p.Forward(y, srcs[i], graph=(j + rep) % 3 != 0)
                s.synchronize()
            except Exception as e:  # surfaced below
                errors.append(e)

        ts = [threading.Thread(target=worker, args=(i,)) for i in range(2)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        torch.cuda.synchronize()
        assert not errors, errors
        for i in range(2):
            for y in outs[i]:
                _check(L, y.cpu().numpy(), xs[i], False, False)
