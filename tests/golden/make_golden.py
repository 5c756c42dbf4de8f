"""Generates tests/golden/known_answers.json.

The reference (CWBudde/algo-fft) ships no stored vectors: its tests build
inputs in code and compare against analytic answers or its naive DFT.  This
script writes those same cases down as data so the oracle and the GPU path
are checked against them:

* analytic known answers, restated from the reference tests cited per case
  (expected values are the closed forms those tests assert);
* the deterministic vectors of plan_reference_test.go (src[i] = (i+1) - 0.5i j)
  with the exact DFT evaluated in 50-digit arithmetic (mpmath), i.e. the
  value the reference's NaiveDFT approximates;
* the Convolve / ConvolveReal basic cases.

Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import math
import os

import mpmath

mpmath.mp.dps = 50
HERE = os.path.dirname(os.path.abspath(__file__))


def exact_dft(x, inverse=False):
    n = len(x)
    out = []
    sgn = 1 if inverse else -1
    for k in range(n):
        s = mpmath.mpc(0)
        for j, v in enumerate(x):
            s += mpmath.mpc(v[0], v[1]) * mpmath.expjpi(mpmath.mpf(sgn * 2 * ((j * k) % n)) / n)
        if inverse:
            s /= n
        out.append([float(s.real), float(s.imag)])
    return out


def c2c(name, cite, n, x, expect, tol, kind="forward", prec="complex64"):
    return {"name": name, "cite": cite, "kind": kind, "precision": prec, "n": n, "input": x,
            "expected": expect, "tol": tol}


cases = []

# plan_signals_test.go:8-33 TestFFTConstantSignal: ones(16) -> [16, 0, ...], tol 1e-3.
n = 16
cases.append(c2c("constant16", "plan_signals_test.go:8", n, [[1.0, 0.0]] * n,
                 [[float(n), 0.0]] + [[0.0, 0.0]] * (n - 1), 1e-3))

# plan_signals_test.go:35-70 TestFFTPureSinusoid: exp(2πi 3j/32) -> 32 at bin 3, tol 1e-2.
n, k = 32, 3
x = [[math.cos(2 * math.pi * k * j / n), math.sin(2 * math.pi * k * j / n)] for j in range(n)]
x = [[float(mpmath.mpf(a)), float(mpmath.mpf(b))] for a, b in x]
cases.append(c2c("sinusoid32_k3", "plan_signals_test.go:35", n, x,
                 [[float(n), 0.0] if i == k else [0.0, 0.0] for i in range(n)], 1e-2))

# plan_signals_test.go:72-105 TestFFTNyquistFrequency: (+1,-1,...) -> 32 at bin 16.
n = 32
cases.append(c2c("nyquist32", "plan_signals_test.go:72", n, [[1.0 if j % 2 == 0 else -1.0, 0.0] for j in range(n)],
                 [[float(n), 0.0] if i == n // 2 else [0.0, 0.0] for i in range(n)], 1e-2))

# precision_test.go:318-405 testLargePrecision: impulse -> all ones, complex128, tol 1e-11
# (sizes 65536..262144 there; the fixture keeps the rule and a small n, the GPU test
# rebuilds the large sizes from the rule).
for n in (8, 1024):
    cases.append(c2c(f"impulse{n}_c128", "precision_test.go:336", n, [[1.0, 0.0]] + [[0.0, 0.0]] * (n - 1),
                     [[1.0, 0.0]] * n, 1e-11, prec="complex128"))

# plan_reference_test.go:9-35 TestForwardMatchesReferenceSmall: src[i] = (i+1) - 0.5 i j,
# n = 2..256, tol 5e-3 against NaiveDFT.  Expected = exact DFT.
for n in (2, 4, 8, 16, 32, 64, 128, 256):
    x = [[float(i + 1), -0.5 * i] for i in range(n)]
    cases.append(c2c(f"refvec{n}", "plan_reference_test.go:9", n, x, exact_dft(x), 5e-3))

# plan_reference_test.go:37-62 TestInverseMatchesReferenceSmall: inverse of the DFT, tol 1e-4.
for n in (2, 4, 8, 16):
    x = [[float(i + 1), -0.5 * i] for i in range(n)]
    X = exact_dft(x)
    cases.append(c2c(f"refvec_inv{n}", "plan_reference_test.go:37", n, X, exact_dft(X, inverse=True), 1e-4,
                     kind="inverse"))

# plan_real_test.go:14-36 TestPlanRealForwardImpulse: n=16 impulse -> ones(9), tol 1e-5.
cases.append({"name": "real_impulse16", "cite": "plan_real_test.go:14", "kind": "r2c", "precision": "float32",
              "n": 16, "input": [1.0] + [0.0] * 15, "expected": [[1.0, 0.0]] * 9, "tol": 1e-5})
# plan_real_test.go:90-120 TestPlanRealForwardConstant: n=32 of 2.0 -> [64, 0...], tol 1e-4.
cases.append({"name": "real_constant32", "cite": "plan_real_test.go:90", "kind": "r2c", "precision": "float32",
              "n": 32, "input": [2.0] * 32, "expected": [[64.0, 0.0]] + [[0.0, 0.0]] * 16, "tol": 1e-4})
# plan_real_test.go:122-161 TestPlanRealForwardCosine: cos(2π 3 i/32) -> 16 at bin 3, tol 1e-3.
x = [float(mpmath.mpf(math.cos(2 * math.pi * 3 * i / 32))) for i in range(32)]
x = [float(v) for v in x]
cases.append({"name": "real_cosine32_k3", "cite": "plan_real_test.go:122", "kind": "r2c", "precision": "float32",
              "n": 32, "input": x, "expected": [[16.0, 0.0] if i == 3 else [0.0, 0.0] for i in range(17)],
              "tol": 1e-3})

# convolve_test.go:9-25 TestConvolveBasic and convolve_real_test.go:10-27 TestConvolveRealBasic.
cases.append({"name": "convolve_basic", "cite": "convolve_test.go:9", "kind": "convolve", "precision": "complex64",
              "a": [[1.0, 0.0], [2.0, 0.0], [3.0, 0.0]], "b": [[4.0, 0.0], [5.0, 0.0]],
              "expected": [[4.0, 0.0], [13.0, 0.0], [22.0, 0.0], [15.0, 0.0]], "tol": 1e-4})
cases.append({"name": "convolve_real_basic", "cite": "convolve_real_test.go:10", "kind": "convolve_real",
              "precision": "float32", "a": [1.0, 2.0, 3.0], "b": [4.0, 5.0], "expected": [4.0, 13.0, 22.0, 15.0],
              "tol": 1e-3})

with open(os.path.join(HERE, "known_answers.json"), "w") as f:
    json.dump({"generator": "tests/golden/make_golden.py", "cases": cases}, f, indent=0)
print(f"wrote {len(cases)} cases")


# ---- N-D cases (plan_2d_test.go:202-383, plan_3d_test.go:237-380) ----------
# The reference builds its inputs with Go's PCG generator
# (generateRandom2DSignal, plan_2d_test.go:15-26: re and im each
# rng.Float64()*20 - 10, cast to float32).  Go's stream is not reproduced
# here; the fixtures keep the tests' shapes, value distribution (U[-10, 10)
# float32), batch/stride layouts and tolerances, with inputs from numpy's
# seeded generator and expected values from the exact N-D DFT (axis by axis
# in 50-digit arithmetic), i.e. what NaiveDFT2D / NaiveDFT3D approximate.
import numpy as np  # noqa: E402


def exact_dft_nd(x, dims, inverse=False):
    a = np.empty(dims, dtype=object)
    flat = a.reshape(-1)
    for i, v in enumerate(x):
        flat[i] = mpmath.mpc(v[0], v[1])
    for ax, n in enumerate(dims):
        a = np.moveaxis(a, ax, -1)
        out = np.empty_like(a)
        sgn = 1 if inverse else -1
        w = [mpmath.expjpi(mpmath.mpf(sgn * 2 * j) / n) for j in range(n)]
        for idx in np.ndindex(*a.shape[:-1]):
            row = a[idx]
            for k in range(n):
                s = mpmath.mpc(0)
                for j in range(n):
                    s += row[j] * w[(j * k) % n]
                out[idx + (k,)] = s / n if inverse else s
        a = np.moveaxis(out, -1, ax)
    return [[float(v.real), float(v.imag)] for v in a.reshape(-1)]


def nd_input(dims, seed, prec):
    rng = np.random.default_rng(seed)
    n = int(np.prod(dims))
    re = rng.random(n) * 20 - 10
    im = rng.random(n) * 20 - 10
    if prec == "complex64":
        re, im = re.astype(np.float32).astype(np.float64), im.astype(np.float32).astype(np.float64)
    return [[float(a), float(b)] for a, b in zip(re, im)]


nd_cases = []
for dims, kind, prec, tol, cite in (
        [((r, c), "forward", "complex64", 1e-3, "plan_2d_test.go:202") for r, c in
         ((2, 2), (4, 4), (8, 8), (16, 16), (4, 8), (8, 4))] +
        [((r, c), "inverse", "complex64", 1e-3, "plan_2d_test.go:250") for r, c in
         ((2, 2), (4, 4), (8, 8), (16, 16), (4, 8))] +
        [((r, c), "forward", "complex128", 1e-10, "plan_2d_test.go:339") for r, c in ((4, 4), (8, 8), (4, 8))] +
        [(d, "forward", "complex64", 1e-2, "plan_3d_test.go:237") for d in
         ((2, 2, 2), (4, 4, 4), (8, 8, 8), (4, 8, 16))] +
        [(d, "forward", "complex128", 1e-9, "plan_3d_test.go:339") for d in ((2, 2, 2), (4, 4, 4), (8, 8, 8))]):
    seed = int(np.prod(dims)) * 7 + len(dims) + (1 if kind == "inverse" else 0) + (2 if prec == "complex128" else 0)
    x = nd_input(dims, seed, prec)
    nd_cases.append({"name": f"{'x'.join(map(str, dims))}_{kind}_{prec}", "cite": cite, "dims": list(dims),
                     "kind": kind, "precision": prec, "input": x, "expected": exact_dft_nd(x, dims, kind == "inverse"),
                     "tol_abs": tol})

# batch + stride layouts: plan_2d_test.go:294-337 (4x4, batch 2, stride 21)
# and plan_3d_test.go:293-330 (2x3x4, batch 2, stride 31), tolerance 1e-3.
for dims, stride, cite in (((4, 4), 21, "plan_2d_test.go:294"), ((2, 3, 4), 31, "plan_3d_test.go:293")):
    sig = [nd_input(dims, 100 + b, "complex64") for b in range(2)]
    nd_cases.append({"name": f"{'x'.join(map(str, dims))}_batch2_stride{stride}", "cite": cite, "dims": list(dims),
                     "kind": "forward_batch", "precision": "complex64", "batch": 2, "stride": stride,
                     "input": sig, "expected": [exact_dft_nd(s, dims) for s in sig], "tol_abs": 1e-3})

with open(os.path.join(HERE, "nd_known_answers.json"), "w") as f:
    json.dump({"generator": "tests/golden/make_golden.py", "cases": nd_cases}, f, indent=0)
