"""The allocation-free batched entry point (gfft_exec_batch_noalloc).

It serves callers that cannot allocate device memory while they run a
transform; its scratch lives in a fixed array inside the library.  Each
check compares it, through the C ABI, with the regular entry point
(gfft_forward_batch / gfft_inverse_batch) on two calls in a row, within the
tolerance of the other parity tests.  This file is named to be collected
last, so a failure here leaves every other test already run."""
import ctypes

import numpy as np
import pytest

import algofft
from helpers import rel_l2, seeded_complex, tol_c2c

pytestmark = pytest.mark.gpu


def _noalloc(plan, direction, dst, src, count):
    import torch
    L = algofft.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return L.gfft_exec_batch_noalloc(plan._h, direction, ctypes.c_void_p(dst.data_ptr()), dst.numel(),
                                     ctypes.c_void_p(src.data_ptr()), src.numel(), count, stream)


@pytest.mark.parametrize("n,prec", [(1 << 16, algofft.COMPLEX64), (1 << 20, algofft.COMPLEX64),
                                    (1 << 21, algofft.COMPLEX64), (1 << 15, algofft.COMPLEX128)])
def test_noalloc_matches_regular_entry_point(n, prec):
    import torch
    c128 = prec == algofft.COMPLEX128
    dtype = np.complex128 if c128 else np.complex64
    count = max(2, (1 << 22) // n)
    # variant pinned to the two-pass kernel (the path this entry point runs)
    tok = next(t for t in algofft.Variants(n, prec) if "-tp-" in t)
    with algofft.Plan(n, prec, variant=tok) as p:
        for call in range(2):  # two calls in a row share the static scratch
            x = seeded_complex(n * count, seed=100 + call, dtype=dtype)
            src = torch.from_numpy(x).cuda()
            want = torch.empty_like(src)
            got = torch.full_like(src, float("nan"))
            for direction in (-1, 1):
                fn = p.ForwardBatch if direction < 0 else p.InverseBatch
                fn(want, src, count)
                assert _noalloc(p, direction, got, src, count) == 0, algofft.lib().gfft_last_error()
                torch.cuda.synchronize()
                p.Check()
                assert rel_l2(got.cpu().numpy(), want.cpu().numpy()) <= tol_c2c(n, c128)


def test_noalloc_rejects_what_it_cannot_hold():
    import torch
    n = 1 << 22  # 32 MiB per complex64 transform: two slots exceed the array
    tok = next(t for t in algofft.Variants(n) if "-tp-" in t)
    with algofft.Plan(n, variant=tok) as p:
        a = torch.zeros(n, dtype=torch.complex64, device="cuda")
        assert _noalloc(p, -1, a, a, 1) == algofft.ErrInvalidArgument.status
        assert b"scratch" in algofft.lib().gfft_last_error()
    with algofft.NewPlan(1024) as p:  # single-pass schedule: not this kernel
        a = torch.zeros(1024, dtype=torch.complex64, device="cuda")
        assert _noalloc(p, -1, a, a, 1) == algofft.ErrNotImplemented.status


@pytest.mark.parametrize("n,count", [(1 << 16, 17), (1 << 16, 3), (1 << 15, 33)])
def test_noalloc_partial_last_group(n, count):
    """Batches that end in a partial group of transforms (the plan groups 16
    transforms of 2^16 points and 32 of 2^15 per scratch slot): the entry
    point against the regular one and against numpy's FP64 FFT, two calls in
    a row."""
    import torch
    tok = next(t for t in algofft.Variants(n) if "-tp-" in t)
    with algofft.Plan(n, variant=tok) as p:
        for call in range(2):
            x = seeded_complex(n * count, seed=200 + call)
            src = torch.from_numpy(x).cuda()
            want = torch.empty_like(src)
            got = torch.full_like(src, float("nan"))
            p.ForwardBatch(want, src, count)
            assert _noalloc(p, -1, got, src, count) == 0, algofft.lib().gfft_last_error()
            torch.cuda.synchronize()
            p.Check()
            g = got.cpu().numpy()
            assert rel_l2(g, want.cpu().numpy()) <= tol_c2c(n, False)
            ref = np.fft.fft(x.astype(np.complex128).reshape(count, n), axis=1)
            assert rel_l2(g.reshape(count, n), ref) <= tol_c2c(n, False)
