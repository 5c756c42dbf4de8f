"""The N > 1 path on CPU: two gloo ranks shard a batch by transform index
(no exchange step), each transforms its slice, and the job's time is the
max over ranks.  The oracle stands in for the GPU transform (CPU test)."""
import os
import socket
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, n, count, out_dir):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import bench
    import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(0)
        x = (rng.standard_normal(n * count) + 1j * rng.standard_normal(n * count)).astype(np.complex64)
        lo, hi = bench.shard(count, rank, world)
        y = oracle.batch(x[lo * n:hi * n], n)
        parts = [None] * world
        dist.all_gather_object(parts, (lo, hi, y))
        t = bench.max_over_ranks(1.5 + rank, dist)
        if rank == 0:
            np.save(os.path.join(out_dir, "gathered.npy"), np.concatenate([p[2] for p in sorted(parts, key=lambda q: q[0])]))
            np.save(os.path.join(out_dir, "bounds.npy"), np.array([p[:2] for p in parts]))
            np.save(os.path.join(out_dir, "t.npy"), np.array([t]))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding_and_max_time(tmp_path):
    import torch.multiprocessing as mp
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import bench  # noqa: F401  (importable without a GPU)
    import oracle
    n, count, world = 64, 37, 2
    mp.spawn(_worker, args=(world, _free_port(), n, count, str(tmp_path)), nprocs=world, join=True)
    rng = np.random.default_rng(0)
    x = (rng.standard_normal(n * count) + 1j * rng.standard_normal(n * count)).astype(np.complex64)
    whole = oracle.batch(x, n)
    got = np.load(tmp_path / "gathered.npy")
    assert np.array_equal(got, whole)  # sharding by transform index is exact
    b = np.load(tmp_path / "bounds.npy")
    assert b[0][0] == 0 and b[-1][1] == count and all(b[i][1] == b[i + 1][0] for i in range(world - 1))
    assert float(np.load(tmp_path / "t.npy")[0]) == 2.5  # max over ranks
