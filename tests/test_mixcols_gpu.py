"""Parity of the compiled mixed-radix column tiles (k_mix_cols) with numpy's
FP64 FFT: the four-step of 7-smooth lengths whose two factors both have a
compiled schedule (every 7-smooth column length 48..1024), forward and
inverse, both precisions, against the runtime-radix two-pass of the same
length, and as the column passes of N-D plans and strided column batches.
The reference runs these lengths through its mixed-radix recursion
(internal/fft/mixedradix.go:45-188)."""
import numpy as np
import pytest

import algofft
from helpers import rel_l2, seeded_complex, tol_c2c

pytestmark = pytest.mark.gpu

# Two-pass 7-smooth lengths: odd factors (partial tiles in both passes),
# factors whose radices divide (147 = 21 x 7, 343 = 49 x 7) and do not
# (250 = 25 x 10; 120 = 12 x 10 and 756 = 28 x 27 on a thread per
# larger-radix butterfly), the largest factors (1000, 1008).
MIXC = [13440, 21609, 33075, 36750, 50421, 62500, 100000, 117649, 240000, 571536, 1000000, 1008000]


def _mixc_token(n, prec=0):
    toks = [t for t in algofft.Variants(n, prec) if "-mixc-" in t]
    assert toks, (n, algofft.Variants(n, prec))
    a, b = (int(v) for v in toks[0].rsplit("-", 1)[1].split("x"))
    assert a * b == n and 48 <= a <= b <= 1024
    return toks[0]


def _run(plan, x, count, inverse=False, inplace=False):
    import torch
    src = torch.from_numpy(x).cuda()
    dst = src if inplace else torch.empty_like(src)
    (plan.InverseBatch if inverse else plan.ForwardBatch)(dst, src, count)
    torch.cuda.synchronize()
    plan.Check()
    return dst.cpu().numpy()


@pytest.mark.parametrize("n", MIXC)
def test_mixc_c64(n):
    count = max(1, min(4, (1 << 21) // n))
    x = seeded_complex(n * count, seed=n % 10007)
    tok = _mixc_token(n)
    with algofft.NewPlan(n) as p:
        assert p.Algorithm() == tok  # the default schedule for these lengths
    with algofft.Plan(n, variant=tok) as p:
        y = _run(p, x, count)
        back = _run(p, y, count, inverse=True)
    ref = np.fft.fft(x.astype(np.complex128).reshape(count, n), axis=1).ravel()
    assert rel_l2(y, ref) <= tol_c2c(n, False)
    assert rel_l2(back, x) <= 2 * tol_c2c(n, False)


@pytest.mark.parametrize("n", [8000, 21609, 50421, 100000, 240000, 571536, 1000000])
def test_mixc_c128(n):
    count = 2
    x = seeded_complex(n * count, seed=n % 10007, dtype=np.complex128)
    tok = _mixc_token(n, 1)
    with algofft.Plan(n, algofft.COMPLEX128, variant=tok) as p:
        y = _run(p, x, count)
        back = _run(p, y, count, inverse=True)
    ref = np.fft.fft(x.reshape(count, n), axis=1).ravel()
    assert rel_l2(y, ref) <= tol_c2c(n, True)
    assert rel_l2(back, x) <= 2 * tol_c2c(n, True)


@pytest.mark.parametrize("n", [50421, 100000])
def test_mixc_matches_runtime_two_pass_and_in_place(n):
    count = 3
    x = seeded_complex(n * count, seed=3)
    rt = [t for t in algofft.Variants(n) if "-mixed2-" in t]
    assert rt
    with algofft.Plan(n, variant=_mixc_token(n)) as p:
        a = _run(p, x, count)
        inplace = _run(p, x, count, inplace=True)
    with algofft.Plan(n, variant=rt[0]) as p:
        b = _run(p, x, count)
    np.testing.assert_array_equal(a, inplace)
    assert rel_l2(a, b) <= 2 * tol_c2c(n, False)


@pytest.mark.parametrize("dims", [(343, 96), (147, 5, 16), (1000, 24), (250, 3)])
def test_mixc_nd_column_axes(dims):
    """The leading axes run as column batches (rows `inner` apart) through
    the compiled tiles, partial tiles included."""
    import torch
    x = seeded_complex(int(np.prod(dims)), seed=len(dims))
    with algofft.NewPlanND(list(dims)) as p:
        src = torch.from_numpy(x).cuda()
        dst = torch.empty_like(src)
        p.Forward(dst, src)
        back = torch.empty_like(src)
        p.Inverse(back, dst)
        torch.cuda.synchronize()
        y, b = dst.cpu().numpy(), back.cpu().numpy()
    ref = np.fft.fftn(x.reshape(dims).astype(np.complex128)).ravel()
    tol = 1.5 * tol_c2c(int(np.prod(dims)), False)
    assert rel_l2(y, ref) <= tol
    assert rel_l2(b, x) <= 2 * tol


@pytest.mark.parametrize("n,cols,stride", [(343, 40, 40), (400, 16, 100), (147, 3, 7)])
def test_mixc_strided_columns(n, cols, stride):
    """count adjacent transforms with rows `stride` apart (the column form of
    gfft_exec_strided_batch) against numpy per column."""
    import torch
    total = (n - 1) * stride + cols
    x = seeded_complex(total, seed=n)
    with algofft.NewPlan(n) as p:
        src = torch.from_numpy(x).cuda()
        dst = torch.zeros_like(src)
        p.StridedBatch(dst, src, cols, stride, 1)
        torch.cuda.synchronize()
        got = dst.cpu().numpy()
    for c in range(cols):
        ref = np.fft.fft(x[c::stride][:n].astype(np.complex128))
        assert rel_l2(got[c::stride][:n], ref) <= tol_c2c(n, False), c


# one-pass compiled schedules (rows mode): several whole transforms per CTA;
# lengths with both thread layouts, the smallest and largest table lengths,
# three-stage schedules (1080 = 12 x 10 x 9 .. 12000 = 25 x 24 x 20;
# complex128 up to 6144)
ROWS = [48, 60, 100, 120, 147, 343, 500, 756, 1000, 1024, 1080, 2000, 6000, 6561, 10000, 12000]


@pytest.mark.parametrize("n", ROWS)
@pytest.mark.parametrize("c128", [False, True])
def test_mixr_one_pass(n, c128):
    if c128 and n > 6144:
        pytest.skip("complex128 three-stage rows stop at 6144")
    dt = np.complex128 if c128 else np.complex64
    prec = algofft.COMPLEX128 if c128 else algofft.COMPLEX64
    count = 37 if n <= 2000 else 5  # not a multiple of the transforms per CTA: a partial last CTA
    x = seeded_complex(n * count, seed=n, dtype=dt)
    tok = f"gpu-sm100-mixr-n{n}"
    if n & (n - 1):  # powers of two keep their own single-pass kernel (the token still builds)
        assert tok in algofft.Variants(n, prec)
        with algofft.Plan(n, prec) as p:
            assert p.Algorithm() == tok
    with algofft.Plan(n, prec, variant=tok) as p:
        y = _run(p, x, count)
        back = _run(p, y, count, inverse=True)
        inplace = _run(p, x, count, inplace=True)
    ref = np.fft.fft(x.astype(np.complex128).reshape(count, n), axis=1).ravel()
    assert rel_l2(y, ref) <= tol_c2c(n, c128)
    assert rel_l2(back, x) <= 2 * tol_c2c(n, c128)
    np.testing.assert_array_equal(y, inplace)


def test_mixr_batch_distance():
    """Transforms dist > n apart: each read and written at its own offset,
    the gaps left alone."""
    import torch
    n, count, dist = 360, 9, 360 + 13
    x = seeded_complex(dist * count, seed=4)
    with algofft.Plan(n, variant="gpu-sm100-mixr-n360") as p:
        src = torch.from_numpy(x).cuda()
        dst = torch.zeros_like(src)
        p.StridedBatch(dst, src, count, 1, dist)
        torch.cuda.synchronize()
        got = dst.cpu().numpy()
    for b in range(count):
        ref = np.fft.fft(x[b * dist:b * dist + n].astype(np.complex128))
        assert rel_l2(got[b * dist:b * dist + n], ref) <= tol_c2c(n, False)
        assert not np.any(got[b * dist + n:(b + 1) * dist])
