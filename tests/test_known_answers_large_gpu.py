"""The reference's known-answer signals at every schedule class and at large
lengths, where its own tests stop at 1024-262144 points.  The closed forms
hold at any length, so each GPU result is checked against the exact answer
(no FFT on either side):

  - impulse at position p -> X[k] = exp(-2 pi i k p / n)
    (precision_test.go:318-405 uses p = 0: all ones);
  - constant c -> X[0] = n c, zero elsewhere (plan_signals_test.go:8-40);
  - tone exp(2 pi i b j / n) -> n at bin b, zero elsewhere
    (plan_signals_test.go:42-79);
  - alternating +1, -1 (even n) -> n at bin n/2 (plan_signals_test.go:81-121);
  - sin / cos at frequency f -> -i n/2 / n/2 at bin f and their conjugate
    pair at n - f (precision_test.go:415-505).

Each length runs one batch whose rows are these signals.  Every element
is held to the larger of the reference test's own absolute tolerance (1e-3)
and 1e-6 * log2(m) * max(||x||_2, max_k |X_k|) (the stated complex64 bound
applied to the input's norm, or to the largest output where a bin gathers
the whole signal), and every row to the stated relative-L2 bound against
the closed form; m is the FFT length the plan runs (NextPow2(2n - 1) for Bluestein,
whose two FFTs double the bound, as in the other Bluestein tests)."""
import math

import numpy as np
import pytest

import algofft
from helpers import tol_c2c

pytestmark = pytest.mark.gpu

# power-of-two schedules (single pass, two-pass, three-pass), 7-smooth
# single-CTA and two-pass, Bluestein single-kernel and two-pass (the host
# holds the inputs and exact spectra in complex128: 2^21 points at most)
LENGTHS = [2048, 16384, 1 << 15, 1 << 18, 1 << 20, 1 << 21, 1000, 6000, 50421, 100000, 8191, 16411, 65521]


def _rows(n: int):
    """(name, input, exact spectrum) rows, complex128."""
    k = np.arange(n, dtype=np.int64)
    rows = []
    for p in (0, n // 3 + 1):
        x = np.zeros(n, np.complex128)
        x[p] = 1.0
        rows.append((f"impulse@{p}", x, np.exp(-2j * np.pi * ((k * p) % n) / n)))
    c = 0.75 - 0.25j
    X = np.zeros(n, np.complex128)
    X[0] = n * c
    rows.append(("constant", np.full(n, c), X))
    b = 7 % n
    X = np.zeros(n, np.complex128)
    X[b] = n
    rows.append((f"tone@{b}", np.exp(2j * np.pi * ((b * k) % n) / n), X))
    if n % 2 == 0:
        X = np.zeros(n, np.complex128)
        X[n // 2] = n
        rows.append(("nyquist", np.where(k % 2 == 0, 1.0, -1.0).astype(np.complex128), X))
    f = 10
    ang = 2 * np.pi * ((f * k) % n) / n
    X = np.zeros(n, np.complex128)
    X[f], X[n - f] = -0.5j * n, 0.5j * n
    rows.append(("sine", np.sin(ang).astype(np.complex128), X))
    X = np.zeros(n, np.complex128)
    X[f], X[n - f] = 0.5 * n, 0.5 * n
    rows.append(("cosine", np.cos(ang).astype(np.complex128), X))
    return rows


@pytest.mark.parametrize("n", LENGTHS)
def test_known_answers_at_scale(n):
    import torch
    rows = _rows(n)
    x = np.concatenate([r[1] for r in rows]).astype(np.complex64)
    with algofft.NewPlan(n) as p:
        src = torch.from_numpy(x).cuda()
        y = torch.empty_like(src)
        p.ForwardBatch(y, src, len(rows))
        torch.cuda.synchronize()
        got = y.cpu().numpy().astype(np.complex128).reshape(len(rows), n)
        alg = p.Algorithm()
    bluestein = alg.startswith("gpu-sm100-bluestein")
    m = 1 << (2 * n - 2).bit_length() if bluestein else n
    factor = 2.0 if bluestein else 1.0
    for (name, xin, want), g in zip(rows, got):
        xin32 = xin.astype(np.complex64).astype(np.complex128)  # the input the GPU saw
        # rounding grows with the input's norm, and at a bin that gathers
        # the whole signal (a tone, a constant) with that bin's magnitude
        size = max(np.linalg.norm(xin32), np.max(np.abs(want)))
        bound = max(1e-3, factor * 1e-6 * math.log2(m) * size)
        err = np.max(np.abs(g - want))
        assert err <= bound, (alg, name, err, bound)
        rel = np.linalg.norm(g - want) / np.linalg.norm(want)
        assert rel <= factor * tol_c2c(m, False), (alg, name, rel)


@pytest.mark.parametrize("n", [4096, 1 << 16, 1 << 20, 50421, 16411])
def test_known_answers_at_scale_c128(n):
    """The same signals in complex128 against the 1e-13 * log2 N bound."""
    import torch
    rows = _rows(n)
    x = np.concatenate([r[1] for r in rows])
    with algofft.NewPlan64(n) as p:
        src = torch.from_numpy(x).cuda()
        y = torch.empty_like(src)
        p.ForwardBatch(y, src, len(rows))
        torch.cuda.synchronize()
        got = y.cpu().numpy().reshape(len(rows), n)
        alg = p.Algorithm()
    bluestein = alg.startswith("gpu-sm100-bluestein")
    m = 1 << (2 * n - 2).bit_length() if bluestein else n
    factor = 2.0 if bluestein else 1.0
    for (name, xin, want), g in zip(rows, got):
        size = max(np.linalg.norm(xin), np.max(np.abs(want)))
        err = np.max(np.abs(g - want))
        assert err <= factor * 1e-13 * math.log2(m) * size, (alg, name, err)
        assert np.linalg.norm(g - want) / np.linalg.norm(want) <= factor * tol_c2c(m, True), (alg, name)


@pytest.mark.parametrize("n", [4096, 1 << 16, 1 << 20, 6000, 100000])
def test_known_answers_real_at_scale(n):
    """R2C of the reference's real signals (plan_real_test.go:14-161:
    impulse -> all ones, constant c -> n c at bin 0, cos(2 pi f j / n) ->
    n/2 at bin f) at large n, checked bin by bin against the closed forms,
    then C2R back to the signal."""
    import torch
    k = np.arange(n, dtype=np.int64)
    h = n // 2 + 1
    f = 10
    sigs, specs = [], []
    x = np.zeros(n)
    x[0] = 1.0
    sigs.append(("impulse", x))
    specs.append(np.ones(h, np.complex128))
    sigs.append(("constant", np.full(n, 2.0)))
    X = np.zeros(h, np.complex128)
    X[0] = 2.0 * n
    specs.append(X)
    sigs.append(("cosine", np.cos(2 * np.pi * ((f * k) % n) / n)))
    X = np.zeros(h, np.complex128)
    X[f] = n / 2
    specs.append(X)
    xr = np.concatenate([s[1] for s in sigs]).astype(np.float32)
    with algofft.NewPlanRealWithOptions(n, algofft.PlanOptions(Batch=len(sigs))) as p:
        src = torch.from_numpy(xr).cuda()
        spec = torch.empty(len(sigs) * h, dtype=torch.complex64, device="cuda")
        p.Forward(spec, src)
        back = torch.empty_like(src)
        p.Inverse(back, spec)
        torch.cuda.synchronize()
        got = spec.cpu().numpy().astype(np.complex128).reshape(len(sigs), h)
        rt = back.cpu().numpy().astype(np.float64).reshape(len(sigs), n)
    for (name, xin), want, g, r in zip(sigs, specs, got, rt):
        size = max(np.linalg.norm(xin), np.max(np.abs(want)))
        err = np.max(np.abs(g - want))
        assert err <= max(1e-3, 2e-6 * math.log2(n) * size), (name, err)
        assert np.max(np.abs(r - xin)) <= max(1e-5, 4e-6 * math.log2(n) * np.max(np.abs(xin))), name
