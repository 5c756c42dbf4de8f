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
