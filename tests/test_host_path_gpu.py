"""The Go-slice path (gfft_*_host: host arrays, copies inside the call,
plan.go:504-530) against the device-buffer path, for pageable arrays (as a
Go []complex64 arrives; staged through the library's pinned lanes) and
pinned ones, over batches that span several chunks with a partial last
one, in place and out of place."""
import numpy as np
import pytest

import algofft
from helpers import seeded_complex

pytestmark = pytest.mark.gpu


def _device_result(p, x, count, inverse):
    import torch
    src = torch.from_numpy(x).cuda()
    dst = torch.empty_like(src)
    (p.InverseBatch if inverse else p.ForwardBatch)(dst, src, count)
    torch.cuda.synchronize()
    return dst.cpu().numpy()


@pytest.mark.parametrize("n,count", [(4096, 3 * 1024 + 77), (1 << 16, 130), (1 << 20, 9), (1000, 5)])
@pytest.mark.parametrize("pinned", [False, True])
def test_host_slices_equal_device_buffers(n, count, pinned):
    import torch
    x = seeded_complex(n * count, seed=n + count)
    with algofft.NewPlan(n) as p:
        want_f = _device_result(p, x, count, False)
        want_b = _device_result(p, want_f, count, True)
        want_ff = _device_result(p, want_f, count, False)
        if pinned:
            hx_t = torch.from_numpy(x).pin_memory()
            hy_t = torch.empty_like(hx_t).pin_memory()
            hx, hy = hx_t.numpy(), hy_t.numpy()
        else:
            hx, hy = x.copy(), np.empty_like(x)
        p.ForwardBatch(hy, hx, count)
        assert np.array_equal(hy, want_f)
        p.InverseBatch(hx, hy, count)  # into the input array
        assert np.array_equal(hx, want_b)
        p.ForwardBatch(hy, hy, count)  # in place
        assert np.array_equal(hy, want_ff)


def test_host_single_transform():
    x = seeded_complex(2048, seed=4)
    with algofft.NewPlan(2048) as p:
        y = np.empty_like(x)
        p.Forward(y, x)
        assert np.array_equal(y, _device_result(p, x, 1, False))
