"""The CPU oracle pinned against the reference's known answers (committed
fixtures) and against numpy's pocketfft.  CPU only."""
import json
import os

import numpy as np
import pytest

import oracle as O
from helpers import rel_l2, seeded_complex, tol_c2c

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))["cases"]


def _cx(v, dtype):
    return np.array([complex(a, b) for a, b in v], dtype=dtype)


@pytest.mark.parametrize("case", [c for c in GOLDEN if c["kind"] in ("forward", "inverse")], ids=lambda c: c["name"])
def test_oracle_c2c_known_answers(case):
    dtype = np.complex128 if case["precision"] == "complex128" else np.complex64
    x = _cx(case["input"], dtype)
    want = _cx(case["expected"], np.complex128)
    inv = case["kind"] == "inverse"
    # the FP64 arbiter
    got = O.naive_dft(x, inverse=inv)
    assert np.max(np.abs(got - want)) <= case["tol"]
    # the reference's own NaiveDFT formula
    got = O.naive_dft_ref(x, inverse=inv)
    assert np.max(np.abs(got - want)) <= case["tol"]
    # the restated reference Plan path (ForwardBatch with count=1)
    got = O.batch(x, case["n"], inverse=inv)
    assert np.max(np.abs(got.astype(np.complex128) - want)) <= case["tol"]


@pytest.mark.parametrize("case", [c for c in GOLDEN if c["kind"] == "r2c"], ids=lambda c: c["name"])
def test_oracle_real_known_answers(case):
    x = np.array(case["input"], np.float32)
    want = _cx(case["expected"], np.complex128)
    got = O.real_forward(x, case["n"])
    assert np.max(np.abs(got - want)) <= case["tol"]


@pytest.mark.parametrize("case", [c for c in GOLDEN if c["kind"].startswith("convolve")], ids=lambda c: c["name"])
def test_oracle_convolve_known_answers(case):
    if case["kind"] == "convolve":
        got = O.convolve(_cx(case["a"], np.complex64), _cx(case["b"], np.complex64))
        want = _cx(case["expected"], np.complex128)
    else:
        got = O.convolve_real(np.array(case["a"], np.float32), np.array(case["b"], np.float32))
        want = np.array(case["expected"])
    assert np.max(np.abs(got - want)) <= case["tol"]


@pytest.mark.parametrize("n", [1, 2, 3, 5, 7, 12, 16, 60, 97, 128, 1000, 1009, 1024, 4096])
def test_naive_dft_matches_pocketfft(n):
    x = seeded_complex(n, seed=n, dtype=np.complex128)
    assert rel_l2(O.naive_dft(x), np.fft.fft(x)) < 1e-14
    assert rel_l2(O.naive_dft(x, inverse=True), np.fft.ifft(x)) < 1e-14


# One size per reference strategy: DIT codelet range, packed Stockham, six-step,
# 2/3/5 mixed radix, Bluestein (prime and 7-smooth).
@pytest.mark.parametrize("n,algo", [(1024, O.ALGO_DIT), (16384, O.ALGO_DIT), (32768, O.ALGO_STOCKHAM),
                                    (65536, O.ALGO_STOCKHAM), (262144, O.ALGO_SIXSTEP), (1000, O.ALGO_MIXED),
                                    (3 * 5 * 256, O.ALGO_MIXED), (1009, O.ALGO_BLUESTEIN),
                                    (7 * 64, O.ALGO_BLUESTEIN)])
def test_oracle_paths_match_pocketfft(n, algo):
    assert O.algorithm(n) == algo
    x = seeded_complex(n, seed=7)
    ref = np.fft.fft(x.astype(np.complex128))
    y = O.batch(x, n)
    assert rel_l2(y, ref) < tol_c2c(n, False)
    back = O.batch(y, n, inverse=True)
    assert rel_l2(back, x) < 2 * tol_c2c(n, False)
    y2 = O.batch(x.astype(np.complex128), n)
    # complex128 Bluestein follows the reference's unreduced chirp angle
    # (bluestein.go:23-29), whose error grows with n; the others meet 1e-13*log2N.
    lim = 1e-10 if algo == O.ALGO_BLUESTEIN else tol_c2c(n, True)
    assert rel_l2(y2, ref) < lim


def test_oracle_batch_is_per_transform():
    n, count = 256, 9
    x = seeded_complex(n * count, seed=3)
    y = O.batch(x, n, nthreads=4)
    for i in range(count):
        assert np.array_equal(y[i * n:(i + 1) * n], O.batch(x[i * n:(i + 1) * n], n))


@pytest.mark.parametrize("n", [2, 4, 16, 4096, 6, 30])
def test_oracle_real_roundtrip(n):
    rng = np.random.default_rng(n)
    x = rng.uniform(-1, 1, n).astype(np.float32)
    X = O.real_forward(x, n)
    assert rel_l2(X, np.fft.rfft(x.astype(np.float64))) < tol_c2c(n, False)
    assert rel_l2(O.real_inverse(X, n), x) < 2 * tol_c2c(n, False)


def test_oracle_real_invalid_spectrum():
    X = np.zeros(9, np.complex64)
    X[0] = 1 + 1j  # DC must be real (plan_real_generic.go:301-316)
    with pytest.raises(RuntimeError):
        O.real_inverse(X, 16)


def test_oracle_convolve_random():
    rng = np.random.default_rng(11)
    a = rng.uniform(-1, 1, 300).astype(np.float32)
    b = rng.uniform(-1, 1, 41).astype(np.float32)
    assert rel_l2(O.convolve_real(a, b), np.convolve(a.astype(np.float64), b.astype(np.float64))) < 1e-5
    ac = seeded_complex(100, 1)
    bc = seeded_complex(17, 2)
    assert rel_l2(O.convolve(ac, bc), np.convolve(ac.astype(np.complex128), bc.astype(np.complex128))) < 1e-5
