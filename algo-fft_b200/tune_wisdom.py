"""Autotunes the compiled kernel variants on the current GPU and writes the
winners as a wisdom file (the reference's size:precision:features:algorithm:ts
format, wisdom.go), which libgfft.so loads by default from
algo-fft_b200/wisdom/b200_sm100.wisdom.

    python algo-fft_b200/tune_wisdom.py [--out PATH] [--min 2] [--max 16777216] [--iters 10]
"""
from __future__ import annotations

import argparse
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import algofft  # noqa: E402


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "wisdom", "b200_sm100.wisdom"))
    ap.add_argument("--min", type=int, default=2)
    ap.add_argument("--max", type=int, default=1 << 24)
    ap.add_argument("--iters", type=int, default=10)
    ap.add_argument("--batch-mib", type=int, default=512, help="bytes per timed batch")
    ap.add_argument("--report", default="", help="also write the per-variant timings (JSON lines)")
    a = ap.parse_args()
    algofft.ClearWisdom()
    reports = []
    for prec, es in ((algofft.COMPLEX64, 8), (algofft.COMPLEX128, 16)):
        n = max(2, a.min)
        while n <= a.max:
            if len(algofft.Variants(n, prec)) > 1:
                count = max(1, (a.batch_mib << 20) // (es * n))
                rep = algofft.Autotune(n, prec, count=count, iters=a.iters)
                reports.append(rep)
                print(json.dumps(rep), flush=True)
            n *= 2
    os.makedirs(os.path.dirname(a.out), exist_ok=True)
    algofft.ExportWisdom(a.out)
    if a.report:
        with open(a.report, "w") as f:
            for r in reports:
                f.write(json.dumps(r) + "\n")
    print(f"wrote {algofft.WisdomLen()} entries to {a.out}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
