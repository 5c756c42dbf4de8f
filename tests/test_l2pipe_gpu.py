"""The L2-pipelined two-pass schedule (k_l2p: both passes in one persistent
launch, the intermediate in L2-resident scratch slots, per-group completion
counters) against numpy's FP64 FFT, for every compiled split and tile shape:
batches that end in a partial group, a single transform, more groups than
slots, the inverse, in place, a batch distance the copy engine cannot use
(the split-kernel fallback), and agreement with the split two-pass kernels
of the same split."""
import numpy as np
import pytest

import algofft
from helpers import rel_l2, seeded_complex, tol_c2c

pytestmark = pytest.mark.gpu


def _l2p_tokens(n, prec=algofft.COMPLEX64):
    return [t for t in algofft.Variants(n, prec) if "-l2p-" in t]


def _ref(x, n, count, inverse=False):
    a = x.astype(np.complex128).reshape(count, n)
    return (np.fft.ifft(a, axis=1) if inverse else np.fft.fft(a, axis=1)).ravel()


SIZES = [1 << k for k in range(15, 21)]


@pytest.mark.parametrize("n", SIZES)
def test_l2pipe_every_variant(n):
    import torch
    toks = _l2p_tokens(n)
    assert toks, f"no L2-pipelined variant for {n}"
    # 3 groups of 8 MB and a partial fourth (g8 tokens), or one partial group
    count = max(3, (3 * (8 << 20)) // (8 * n) + 1)
    count = min(count, max(3, (1 << 26) // (8 * n)))
    x = seeded_complex(n * count, seed=n % 1000)
    want = _ref(x, n, count)
    src = torch.from_numpy(x).cuda()
    for tok in toks:
        with algofft.Plan(n, variant=tok) as p:
            assert p.Algorithm() == tok
            y = torch.full_like(src, float("nan"))
            p.ForwardBatch(y, src, count)
            torch.cuda.synchronize()
            p.Check()
            assert rel_l2(y.cpu().numpy(), want) <= tol_c2c(n, False), tok


@pytest.mark.parametrize("n", [1 << 15, 1 << 18, 1 << 20])
def test_l2pipe_inverse_in_place_single_and_fallback(n):
    import torch
    tok = _l2p_tokens(n)[-1]
    count = max(2, (1 << 24) // n)
    x = seeded_complex(n * count, seed=7)
    with algofft.Plan(n, variant=tok) as p:
        # inverse, in place
        t = torch.from_numpy(x).cuda()
        p.InverseBatch(t, t, count)
        torch.cuda.synchronize()
        p.Check()
        assert rel_l2(t.cpu().numpy(), _ref(x, n, count, True)) <= tol_c2c(n, False)
        # one transform
        one = torch.from_numpy(x[:n].copy()).cuda()
        y1 = torch.empty_like(one)
        p.Forward(y1, one)
        torch.cuda.synchronize()
        assert rel_l2(y1.cpu().numpy(), _ref(x[:n], n, 1)) <= tol_c2c(n, False)
        # an odd batch distance (16-byte rule of the copy engine): split kernels
        src = torch.zeros(count * (n + 1), dtype=torch.complex64, device="cuda")
        src.view(count, n + 1)[:, :n] = torch.from_numpy(x.reshape(count, n)).cuda()
        dst = torch.zeros_like(src)
        p.StridedBatch(dst, src, count, 1, n + 1)
        torch.cuda.synchronize()
        got = dst.view(count, n + 1)[:, :n].cpu().numpy().ravel()
        assert rel_l2(got, _ref(x, n, count)) <= tol_c2c(n, False)


@pytest.mark.parametrize("n", [1 << 16, 1 << 20])
def test_l2pipe_equals_split_kernels_of_the_same_split(n):
    """Same split, same stage schedule per column: the same arithmetic, so
    the results agree to rounding of the stage order (not bit-exact: the
    tile shapes differ)."""
    import torch
    count = max(2, (1 << 23) // n)
    x = seeded_complex(n * count, seed=3)
    src = torch.from_numpy(x).cuda()
    tok = _l2p_tokens(n)[0]
    split = tok.split("-l2p-")[1].split("-c")[0]
    tp = next(t for t in algofft.Variants(n) if t.startswith(f"gpu-sm100-tp-{split}-"))
    outs = []
    for t in (tok, tp):
        with algofft.Plan(n, variant=t) as p:
            y = torch.empty_like(src)
            p.ForwardBatch(y, src, count)
            torch.cuda.synchronize()
            outs.append(y.cpu().numpy())
    assert rel_l2(outs[0], outs[1]) <= tol_c2c(n, False)
