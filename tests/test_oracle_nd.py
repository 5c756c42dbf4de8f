"""The oracle's N-D restatements (the reference's NaiveDFT2D / NaiveDFT3D
formula, internal/reference/dft2d.go:17-160 and dft3d.go:18-146, and the
exactly reduced FP64 N-D arbiter) against the N-D fixtures (the shapes,
layouts and tolerances of plan_2d_test.go:202-383 and plan_3d_test.go:237-380,
expected values from the exact DFT in 50-digit arithmetic) and numpy."""
import json
import os

import numpy as np
import pytest

import oracle
from helpers import rel_l2

CASES = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "nd_known_answers.json")))["cases"]


def _c(v):
    a = np.asarray(v, dtype=np.float64)
    return a[..., 0] + 1j * a[..., 1]


def _single(c):
    return c["kind"] in ("forward", "inverse")


@pytest.mark.parametrize("case", [c for c in CASES if _single(c)], ids=lambda c: c["name"])
def test_nd_arbiter_and_reference_formula_match_fixtures(case):
    x, want, dims = _c(case["input"]), _c(case["expected"]), case["dims"]
    inverse = case["kind"] == "inverse"
    got = oracle.naive_dft_nd(x, dims, inverse)
    assert rel_l2(got, want) <= 1e-14
    ref = oracle.naive_dft_nd_ref(x, dims, inverse)
    if case["precision"] == "complex64":
        ref = ref.astype(np.complex64)  # the reference's complex64 NaiveDFT2D/3D rounds its sum
    assert np.max(np.abs(ref - want)) <= case["tol_abs"]
    assert rel_l2(ref, want) <= (1e-6 if case["precision"] == "complex64" else 1e-12)


@pytest.mark.parametrize("case", [c for c in CASES if not _single(c)], ids=lambda c: c["name"])
def test_nd_batch_fixtures(case):
    for x, want in zip(case["input"], case["expected"]):
        assert rel_l2(oracle.naive_dft_nd(_c(x), case["dims"]), _c(want)) <= 1e-14


@pytest.mark.parametrize("dims", [(3, 5), (6, 4, 2), (2, 3, 2, 5)])
def test_nd_arbiter_matches_numpy(dims):
    rng = np.random.default_rng(sum(dims))
    x = rng.standard_normal(int(np.prod(dims))) + 1j * rng.standard_normal(int(np.prod(dims)))
    for inverse in (False, True):
        got = oracle.naive_dft_nd(x, dims, inverse)
        want = (np.fft.ifftn if inverse else np.fft.fftn)(x.reshape(dims)).ravel()
        assert rel_l2(got, want) <= 1e-14
