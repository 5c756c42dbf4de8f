"""Writes gfft_constants.cuh: cos/sin(2*pi*j/R) for the in-register DFT
codelets (R = 64 covers every power-of-two radix up to 64; 3, 5 and 7 for the
odd radices; 9 for the composite radix 3 x 3), evaluated with mpmath
cospi/sinpi at 40 digits and rounded to double."""
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
for r in (64, 3, 5, 7, 9):
    out.append(table(f"kCos{r}", r, mpmath.cospi))
    out.append(table(f"kSin{r}", r, mpmath.sinpi))
out.append("}  // namespace gfft\n")
with open(os.path.join(here, "gfft_constants.cuh"), "w") as f:
    f.write("".join(out))
