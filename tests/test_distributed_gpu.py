"""The distributed four-step with its default local transform (the library's
batched device plans on the slab's own device) and its device-side twiddle
product, on one GPU: a world-size-1 NCCL group, so every exchange is the
identity and what runs is the device path of PlanDistributed.  Results are
compared with numpy's FP64 FFT of the whole vector (numpy's FFT is checked
against the oracle's FP64 DFT in test_oracle.py)."""
import numpy as np
import pytest

import algofft
from helpers import rel_l2, tol_c2c

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nccl_world_of_one():
    import torch
    import torch.distributed as dist
    if dist.is_initialized():
        pytest.skip("a process group is already initialized in this process")
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", store=dist.HashStore(), rank=0, world_size=1)
    try:
        yield
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n", [1 << 20, 15360])
@pytest.mark.parametrize("prec", [algofft.COMPLEX64, algofft.COMPLEX128])
def test_distributed_default_device_path(nccl_world_of_one, n, prec):
    import torch
    from algofft.distributed import PlanDistributed
    c128 = prec == algofft.COMPLEX128
    dt = torch.complex128 if c128 else torch.complex64
    rng = np.random.default_rng(11)
    x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex128 if c128 else np.complex64)
    want = np.fft.fft(x.astype(np.complex128))
    with PlanDistributed(n, prec, device="cuda:0") as p:
        slab = torch.from_numpy(x).to("cuda:0", dt)
        y = p.Forward(slab)
        back = p.Inverse(y)
        yt = p.Forward(slab, natural_order=False)
        back_t = p.Inverse(yt, natural_order=False)
        torch.cuda.synchronize()
        assert y.device.type == "cuda" and all(k[1] == 0 for k in p._plans)
        tol = tol_c2c(n, c128)
        assert rel_l2(y.cpu().numpy(), want) <= tol
        # transposed layout: rows k1, columns k2 -> X[k1 + N1 k2]
        assert rel_l2(yt.cpu().numpy().reshape(p.n1, p.n2), want.reshape(p.n2, p.n1).T) <= tol
        assert rel_l2(back.cpu().numpy(), x) <= 2 * tol
        assert rel_l2(back_t.cpu().numpy(), x) <= 2 * tol
