"""Writes gfft_constants.cuh: cos/sin(2*pi*j/R) for the in-register DFT
codelets (R = 64 covers every power-of-two radix up to 64; 3, 5 and 7 for the
odd radices; every other 7-smooth composite radix up to 64 for the twiddles
between its factors), evaluated with mpmath cospi/sinpi at 40 digits and
rounded to double, plus root_cos_tab / root_sin_tab, which select a table by
radix at compile time."""
import os
import mpmath

mpmath.mp.dps = 40
here = os.path.dirname(os.path.abspath(__file__))


def table(name, r, fn):
    vals = []
    for j in range(r):
        v = fn(mpmath.mpf(2 * j) / r)
        vals.append(repr(float(v)))
    body = ",\n    ".join(", ".join(vals[i:i + 4]) for i in range(0, len(vals), 4))
    return f"constexpr double {name}[{r}] = {{\n    {body}}};\n"


out = ["// Generated by gen_constants.py; do not edit.\n#pragma once\n\nnamespace gfft {\n"]


def smooth7(n):
    for p in (2, 3, 5, 7):
        while n % p == 0:
            n //= p
    return n == 1


RADICES = [64] + [r for r in range(3, 65) if smooth7(r) and r & (r - 1)]
for r in RADICES:
    out.append(table(f"kCos{r}", r, mpmath.cospi))
    out.append(table(f"kSin{r}", r, mpmath.sinpi))
for fn, tab in (("root_cos_tab", "kCos"), ("root_sin_tab", "kSin")):
    cases = "".join(f"    case {r}: return {tab}{r}[m];\n" for r in RADICES)
    out.append(f"__host__ __device__ constexpr double {fn}(int r, int m) {{\n  switch (r) {{\n{cases}  }}\n  return 2.0;\n}}\n")
out.append("__host__ __device__ constexpr bool has_root_tab(int r) {\n  return " +
           " || ".join(f"r == {r}" for r in RADICES) + ";\n}\n")
out.append("}  // namespace gfft\n")
with open(os.path.join(here, "gfft_constants.cuh"), "w") as f:
    f.write("".join(out))
