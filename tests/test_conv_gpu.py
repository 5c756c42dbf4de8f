"""Parity of Convolve / Correlate / ConvolveReal (convolve.go, correlate.go,
convolve_real.go) with the oracle and FP64 references."""
import json
import os

import numpy as np
import pytest

import algofft
import oracle as O
from helpers import rel_l2, seeded_complex

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))["cases"]
TOL = 1e-5  # relative L2 of a three-transform chain in float32


@pytest.mark.parametrize("case", [c for c in GOLDEN if c["kind"].startswith("convolve")], ids=lambda c: c["name"])
def test_convolve_known_answers(case):
    if case["kind"] == "convolve":
        a = np.array([complex(*v) for v in case["a"]], np.complex64)
        b = np.array([complex(*v) for v in case["b"]], np.complex64)
        got = np.empty(a.size + b.size - 1, np.complex64)
        algofft.Convolve(got, a, b)
        want = np.array([complex(*v) for v in case["expected"]])
    else:
        a = np.array(case["a"], np.float32)
        b = np.array(case["b"], np.float32)
        got = np.empty(a.size + b.size - 1, np.float32)
        algofft.ConvolveReal(got, a, b)
        want = np.array(case["expected"])
    assert np.max(np.abs(got - want)) <= case["tol"]


@pytest.mark.parametrize("na,nb", [(3, 2), (100, 17), (1000, 9), (1021, 3), (4096, 4097), (7, 1)])
def test_convolve_complex(na, nb):
    a, b = seeded_complex(na, 1), seeded_complex(nb, 2)
    got = np.empty(na + nb - 1, np.complex64)
    algofft.Convolve(got, a, b)
    ref = np.convolve(a.astype(np.complex128), b.astype(np.complex128))
    assert rel_l2(got, ref) <= TOL
    assert rel_l2(got, O.convolve(a, b)) <= 2 * TOL


@pytest.mark.parametrize("na,nb", [(300, 41), (4096, 4097), (1, 1), (65536, 100)])
def test_convolve_real(na, nb):
    rng = np.random.default_rng(na)
    a = rng.uniform(-1, 1, na).astype(np.float32)
    b = rng.uniform(-1, 1, nb).astype(np.float32)
    got = np.empty(na + nb - 1, np.float32)
    algofft.ConvolveReal(got, a, b)
    ref = np.convolve(a.astype(np.float64), b.astype(np.float64))
    assert rel_l2(got, ref) <= TOL
    assert rel_l2(got, O.convolve_real(a, b)) <= 2 * TOL


def test_correlate_and_autocorrelate():
    a, b = seeded_complex(200, 3), seeded_complex(31, 4)
    got = np.empty(230, np.complex64)
    algofft.CrossCorrelate(got, a, b)
    # correlate.go:26-32: convolve with the conjugate reverse of b
    ref = np.convolve(a.astype(np.complex128), np.conj(b[::-1]).astype(np.complex128))
    assert rel_l2(got, ref) <= TOL
    auto = np.empty(399, np.complex64)
    algofft.AutoCorrelate(auto, a)
    ref = np.convolve(a.astype(np.complex128), np.conj(a[::-1]).astype(np.complex128))
    assert rel_l2(auto, ref) <= TOL


def test_convolve128_and_device_path():
    import torch
    a = seeded_complex(500, 5, dtype=np.complex128)
    b = seeded_complex(77, 6, dtype=np.complex128)
    got = np.empty(576, np.complex128)
    algofft.Convolve128(got, a, b)
    assert rel_l2(got, np.convolve(a, b)) <= 1e-12
    ta, tb = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    tg = torch.empty(576, dtype=torch.complex128, device="cuda")
    algofft.Convolve(tg, ta, tb)
    torch.cuda.synchronize()
    assert np.allclose(tg.cpu().numpy(), got, rtol=0, atol=1e-12)


def test_convolve_real_batch_shared_kernel():
    # the convolution workload: signals of 2^20 samples with a 4097-tap kernel
    import torch
    n, taps, count = 1 << 20, 4097, 4
    g = torch.Generator(device="cuda")
    g.manual_seed(1)
    a = torch.rand(count * n, generator=g, device="cuda") * 2 - 1
    b = torch.rand(taps, generator=g, device="cuda") * 2 - 1
    L = n + taps - 1
    dst = torch.empty(count * L, device="cuda")
    algofft.ConvolveRealBatch(dst, a, n, count, b)
    torch.cuda.synchronize()
    F = 1 << 21
    for i in (0, count - 1):
        ai = a[i * n:(i + 1) * n].double()
        ref = torch.fft.irfft(torch.fft.rfft(ai, F) * torch.fft.rfft(b.double(), F), F)[:L]
        got = dst[i * L:(i + 1) * L].double()
        assert (torch.linalg.vector_norm(got - ref) / torch.linalg.vector_norm(ref)).item() <= TOL


@pytest.mark.parametrize("na,nb", [(20000, 1), (50001, 2049), (100000, 8193), (12289, 2), (300000, 4097)])
def test_convolve_real_overlap_save_lengths(na, nb):
    # long signals with short kernels run overlap-save blocks of 2^12..2^15
    # points; the result is the same linear convolution
    rng = np.random.default_rng(na + nb)
    a = rng.uniform(-1, 1, na).astype(np.float32)
    b = rng.uniform(-1, 1, nb).astype(np.float32)
    got = np.empty(na + nb - 1, np.float32)
    algofft.ConvolveReal(got, a, b)
    F = 1 << int(np.ceil(np.log2(na + nb - 1)))
    ref = np.fft.irfft(np.fft.rfft(a.astype(np.float64), F) * np.fft.rfft(b.astype(np.float64), F), F)[:na + nb - 1]
    assert rel_l2(got, ref) <= TOL
    # every output sample, not only the norm: block seams are exact
    assert np.max(np.abs(got - ref)) <= 20 * TOL * np.max(np.abs(ref))


def test_convolve_real_overlap_save_float64_and_strided_batch():
    import torch
    rng = np.random.default_rng(9)
    a = rng.uniform(-1, 1, 70000)
    b = rng.uniform(-1, 1, 300)
    got = np.empty(70299)
    algofft.ConvolveReal(got, a, b)
    assert rel_l2(got, np.convolve(a, b)) <= 1e-12
    # strided batch: signals 70100 apart, outputs 70400 apart
    count, na, ad, dd = 3, 70000, 70100, 70400
    A = torch.from_numpy(rng.uniform(-1, 1, count * ad).astype(np.float32)).cuda()
    K = torch.from_numpy(rng.uniform(-1, 1, 300).astype(np.float32)).cuda()
    D = torch.zeros(count * dd, device="cuda")
    algofft.ConvolveRealBatch(D, A, na, count, K, a_dist=ad, dst_dist=dd)
    torch.cuda.synchronize()
    Ah, Kh, Dh = A.cpu().numpy().astype(np.float64), K.cpu().numpy().astype(np.float64), D.cpu().numpy()
    for i in range(count):
        ref = np.convolve(Ah[i * ad:i * ad + na], Kh)
        assert rel_l2(Dh[i * dd:i * dd + na + 299], ref) <= TOL
        assert np.all(Dh[i * dd + na + 299:(i + 1) * dd] == 0)  # untouched gap


def test_convolve_errors():
    a = np.ones(3, np.complex64)
    with pytest.raises(algofft.ErrLengthMismatch):
        algofft.Convolve(np.empty(3, np.complex64), a, a)
    with pytest.raises(algofft.ErrInvalidLength):
        algofft.Convolve(np.empty(2, np.complex64), a, np.empty(0, np.complex64))
    with pytest.raises(algofft.ErrNilSlice):
        algofft.ConvolveReal(None, np.ones(2, np.float32), np.ones(2, np.float32))
