"""The reference's own CPU-runnable batch, exactly: complex64 C2C, N = 1024,
count = 256, real and imaginary parts i.i.d. U[-1, 1) float32 from seed 0,
ForwardBatch then InverseBatch (plan.go:504-571; the reference's benchmark
of this call is plan_batch_test.go:427-457).

Both results are checked against the oracle's restatement of the
reference's complex64 ForwardBatch (oracle.batch, the 32x32 codelet path of
plan.go:343-368 for N = 1024) and against the FP64 naive DFT (the arbiter),
by relative L2 error (<= 1e-6 * log2 N) and by maximum error relative to the
largest reference magnitude (same bound)."""
import numpy as np
import pytest

import algofft
import oracle
from helpers import rel_l2, tol_c2c

pytestmark = pytest.mark.gpu

N, COUNT = 1024, 256


def config1_input() -> np.ndarray:
    """Re and Im i.i.d. U[-1, 1) float32 from seed 0, interleaved."""
    rng = np.random.default_rng(0)
    re = rng.uniform(-1.0, 1.0, N * COUNT).astype(np.float32)
    im = rng.uniform(-1.0, 1.0, N * COUNT).astype(np.float32)
    return (re + 1j * im).astype(np.complex64)


def max_rel(got, want) -> float:
    got = np.asarray(got, np.complex128)
    want = np.asarray(want, np.complex128)
    return float(np.max(np.abs(got - want)) / np.max(np.abs(want)))


def _naive_rows(x: np.ndarray, inverse: bool) -> np.ndarray:
    rows = x.reshape(COUNT, N)
    return np.concatenate([oracle.naive_dft(r, inverse) for r in rows])


def test_config1_forward_then_inverse():
    import torch
    x = config1_input()
    tol = tol_c2c(N, False)
    with algofft.NewPlan(N) as p:
        src = torch.from_numpy(x).cuda()
        fwd = torch.empty_like(src)
        back = torch.empty_like(src)
        p.ForwardBatch(fwd, src, COUNT)
        p.InverseBatch(back, fwd, COUNT)
        torch.cuda.synchronize()
        f = fwd.cpu().numpy()
        b = back.cpu().numpy()
    # forward against the restated reference path and the FP64 arbiter
    ref_f = oracle.batch(x, N)
    exact_f = _naive_rows(x, False)
    assert rel_l2(ref_f, exact_f) <= tol  # the restatement itself is within the bound
    assert rel_l2(f, ref_f) <= tol and max_rel(f, ref_f) <= tol
    assert rel_l2(f, exact_f) <= tol and max_rel(f, exact_f) <= tol
    # inverse of the GPU spectrum against the same two, and the round trip
    ref_b = oracle.batch(f, N, inverse=True)
    exact_b = _naive_rows(f, True)
    assert rel_l2(b, ref_b) <= tol and max_rel(b, ref_b) <= tol
    assert rel_l2(b, exact_b) <= tol and max_rel(b, exact_b) <= tol
    assert rel_l2(b, x) <= 2 * tol


def test_config1_host_slices_match_device_buffers():
    """The Go-slice path (host arrays, copies inside the call) gives the same
    bits as the device-buffer path on this batch."""
    import torch
    x = config1_input()
    with algofft.NewPlan(N) as p:
        hf = np.empty_like(x)
        hb = np.empty_like(x)
        p.ForwardBatch(hf, x, COUNT)
        p.InverseBatch(hb, hf, COUNT)
        src = torch.from_numpy(x).cuda()
        df = torch.empty_like(src)
        p.ForwardBatch(df, src, COUNT)
        torch.cuda.synchronize()
    assert np.array_equal(hf, df.cpu().numpy())
    assert rel_l2(hb, x) <= 2 * tol_c2c(N, False)
