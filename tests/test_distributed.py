"""The distributed four-step (one transform over the ranks of a group) on
CPU: gloo ranks, all-to-all exchanges, and the row transforms of each step
computed by torch.fft on the CPU in place of the device plans (the exchange
and index logic is what these tests check).  Results are compared with
numpy's FP64 FFT of the whole vector."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rows_fft(x, inverse):
    import torch
    return torch.fft.ifft(x, dim=1) if inverse else torch.fft.fft(x, dim=1)


def _vector(n, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(n) + 1j * rng.standard_normal(n)


def _worker(rank, world, port, n, prec, out_dir):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "algo-fft_b200"))
    import algofft
    from algofft.distributed import PlanDistributed
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dt = torch.complex64 if prec == "c64" else torch.complex128
        x = torch.from_numpy(_vector(n, 5)).to(dt)
        s = n // world
        slab = x[rank * s:(rank + 1) * s].clone()
        p = PlanDistributed(n, algofft.COMPLEX64 if prec == "c64" else algofft.COMPLEX128, local_fft=_rows_fft)
        y = p.Forward(slab)
        back = p.Inverse(y)
        yt = p.Forward(slab, natural_order=False)
        back_t = p.Inverse(yt, natural_order=False)
        parts = [None] * world
        dist.all_gather_object(parts, (rank, y.numpy(), back.numpy(), back_t.numpy(), yt.numpy(), p.n1, p.n2))
        if rank == 0:
            parts.sort(key=lambda q: q[0])
            np.save(os.path.join(out_dir, "y.npy"), np.concatenate([q[1] for q in parts]))
            np.save(os.path.join(out_dir, "back.npy"), np.concatenate([q[2] for q in parts]))
            np.save(os.path.join(out_dir, "back_t.npy"), np.concatenate([q[3] for q in parts]))
            np.save(os.path.join(out_dir, "yt.npy"), np.stack([q[4] for q in parts]))
            np.save(os.path.join(out_dir, "split.npy"), np.array([parts[0][5], parts[0][6]]))
    finally:
        dist.destroy_process_group()


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("n,world,prec", [(4096, 2, "c128"), (15360, 4, "c128"), (1000, 2, "c64"),
                                          (15360, 2, "c64")])
def test_distributed_forward_inverse(tmp_path, n, world, prec):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(world, _free_port(), n, prec, str(tmp_path)), nprocs=world, join=True)
    x = _vector(n, 5)
    if prec == "c64":
        x = x.astype(np.complex64).astype(np.complex128)
    ref = np.fft.fft(x)
    tol = (1e-6 if prec == "c64" else 1e-13) * np.log2(n)
    y = np.load(tmp_path / "y.npy")
    assert _rel(y, ref) <= tol
    assert _rel(np.load(tmp_path / "back.npy"), x) <= 2 * tol
    assert _rel(np.load(tmp_path / "back_t.npy"), x) <= 2 * tol
    # the transposed layout: rank r holds X[k1 + N1 k2] for its k1 rows
    n1, n2 = (int(v) for v in np.load(tmp_path / "split.npy"))
    assert n1 * n2 == n and n1 % world == 0 and n2 % world == 0
    yt = np.load(tmp_path / "yt.npy").reshape(world, n1 // world, n2)
    k1 = np.arange(n1).reshape(world, n1 // world, 1)
    k2 = np.arange(n2).reshape(1, 1, n2)
    assert _rel(yt, ref[k1 + n1 * k2]) <= tol


def test_split_rules():
    sys.path.insert(0, os.path.join(ROOT, "algo-fft_b200"))
    from algofft.distributed import _split
    assert _split(4096, 2) == (64, 64)
    assert _split(15360, 4) == (120, 128)
    assert _split(1000, 2) == (20, 50)
    with pytest.raises(ValueError):
        _split(9, 2)
    with pytest.raises(ValueError):
        _split(2 * 1024, 4096)
