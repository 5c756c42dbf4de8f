"""Learned planner: dataset measurement, training with the library's own MLP
kernels (gfft_mlp_train), model files, and evaluation against exhaustive
measurement.

The cost model scores (shape, variant) pairs (features: gfft_planner_features)
with a predicted log(ns per element); plan creation with
``PlanOptions(Planner=PlannerLearned)`` takes the variant with the smallest
prediction when the wisdom store has no entry.  Exhaustive measurement (the
autotuner) is the fallback and the arbiter: regret = time of the chosen variant
/ time of the fastest measured one.

    python -m algofft.planner collect --count 3500 --out DATA.jsonl   # on a GPU
    python -m algofft.planner refresh [--data DATA.jsonl] --out NEW.jsonl  # re-time changed shapes
    python -m algofft.planner train --data DATA.jsonl --out MODEL.bin
    python -m algofft.planner report [--data DATA.jsonl] [--model MODEL.bin] [--exercise]

The shipped model (wisdom/planner_b200.bin) was trained by `train` on the
first 3,000 shapes of the shipped measurements (wisdom/planner_data.jsonl.gz,
`collect --seed 2024` on a B200); the last 500 are held out.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import struct
import sys
import time

import numpy as np

from ._lib import ErrInvalidArgument, check, lib
from .plan import COMPLEX64, COMPLEX128, Plan, PlanOptions
from .wisdom import ClearWisdom, ExportWisdomToString, ImportWisdomFromString, Variants

HERE = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DEFAULT_MODEL = os.path.join(HERE, "wisdom", "planner_b200.bin")
TRAIN_SHAPES, HELD_OUT_SHAPES = 3000, 500


def sizes() -> tuple[int, int, int]:
    d, h, n = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64()
    lib().gfft_mlp_sizes(ctypes.byref(d), ctypes.byref(h), ctypes.byref(n))
    return d.value, h.value, n.value


def features(prec: int, n: int, batch: int, stride: int, real: int, token: str) -> np.ndarray:
    d, _, _ = sizes()
    out = np.zeros(d, dtype=np.float32)
    check(lib().gfft_planner_features(prec, n, batch, stride, real, token.encode(),
                                      out.ctypes.data_as(ctypes.c_void_p)))
    return out


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal weights, zero biases, in the flat order of include/gfft.h."""
    d, h, n = sizes()
    rng = np.random.default_rng(seed)
    p = np.concatenate([rng.standard_normal(h * d) * math.sqrt(2.0 / d), np.zeros(h),
                        rng.standard_normal(h * h) * math.sqrt(2.0 / h), np.zeros(h),
                        rng.standard_normal(h) * math.sqrt(1.0 / h), [0.0]]).astype(np.float32)
    assert p.size == n
    return p


# ---------------------------------------------------------------- shapes

def smooth7(lo: int, hi: int) -> np.ndarray:
    """7-smooth integers in [lo, hi] that are not powers of two."""
    out = []
    a = 1
    while a <= hi:
        b = a
        while b <= hi:
            c = b
            while c <= hi:
                d = c
                while d <= hi:
                    if d >= lo and d & (d - 1):
                        out.append(d)
                    d *= 7
                c *= 5
            b *= 3
        a *= 2
    return np.array(sorted(out), dtype=np.int64)


def shapes(count: int, seed: int) -> list[dict]:
    """Seeded shapes with at least two candidate variants: 40% powers of two
    2^4..2^22 (2^21 for complex128), 60% 7-smooth lengths log-uniform in
    12..2^21; 25% complex128; 25% the complex child of a real transform;
    2^16..2^24 elements per call."""
    rng = np.random.default_rng(seed)
    sm = smooth7(12, 1 << 21)
    out = []
    while len(out) < count:
        prec = COMPLEX128 if rng.random() < 0.25 else COMPLEX64
        real = int(rng.random() < 0.25)
        if rng.random() < 0.4:
            n = 1 << int(rng.integers(4, 23 - prec))
        else:
            t = rng.uniform(math.log2(12), math.log2((1 << 21) >> prec))
            n = int(sm[min(np.searchsorted(sm, 2 ** t), sm.size - 1)])
        total = int(2 ** rng.uniform(16, 24))
        batch = max(1, total // n)
        if len(Variants(n, prec)) < 2:
            continue
        out.append({"prec": prec, "n": n, "batch": batch, "real": real})
    return out


# ---------------------------------------------------------------- measuring

def _median_ms(fn, iters: int) -> float:
    import torch
    fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(iters):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        ts.append(a.elapsed_time(b))
    return float(np.median(ts))


def _default_token(prec: int, n: int) -> str:
    """The variant the size-class rules pick with an empty wisdom store."""
    with Plan(n, prec) as p:
        name = p.Algorithm()
    if name.startswith("gpu-sm100-bluestein-n"):
        return name.split("-m")[0]
    return name


def measure_shape(s: dict, iters: int = 3) -> dict:
    """Times every variant of the shape (forward, device-resident data)."""
    import torch
    from .real import PlanReal
    prec, n, batch, real = s["prec"], s["n"], s["batch"], s["real"]
    cdt = torch.complex128 if prec == COMPLEX128 else torch.complex64
    rdt = torch.float64 if prec == COMPLEX128 else torch.float32
    times = {}
    if real:
        x = torch.randn(batch * 2 * n, dtype=rdt, device="cuda")
        y = torch.empty(batch * (n + 1), dtype=cdt, device="cuda")
        saved = ExportWisdomToString()
        try:
            for tok in Variants(n, prec):
                ClearWisdom()
                ImportWisdomFromString(f"{n}:{prec}:100:{tok}:0\n")
                with PlanReal(2 * n, prec, PlanOptions(Batch=batch)) as p:
                    times[tok] = _median_ms(lambda: p.Forward(y, x), iters)
        finally:
            ClearWisdom()
            ImportWisdomFromString(saved)
    else:
        x = torch.randn(batch * n, dtype=cdt, device="cuda")
        y = torch.empty_like(x)
        for tok in Variants(n, prec):
            with Plan(n, prec, variant=tok) as p:
                times[tok] = _median_ms(lambda: p.ForwardBatch(y, x, batch), iters)
    saved = ExportWisdomToString()
    ClearWisdom()
    try:
        default = _default_token(prec, n)
    finally:
        ImportWisdomFromString(saved)
    r = dict(s)
    r["times"] = times
    r["default"] = default
    return r


def collect(count: int, seed: int, out: str, iters: int = 3) -> None:
    t0 = time.time()
    with open(out, "w") as f:
        for i, s in enumerate(shapes(count, seed)):
            f.write(json.dumps(measure_shape(s, iters)) + "\n")
            if i % 250 == 0:
                print(f"{i} shapes, {time.time() - t0:.0f} s", file=sys.stderr, flush=True)


def refresh(data: str, out: str, iters: int = 3) -> int:
    """Re-times the shapes of `data` whose candidate set changed since they
    were measured (variants added to or removed from the library), keeps the
    others, and writes the records to `out` in the same order."""
    import gzip
    recs = load_records(data)
    n_new = 0
    opener = gzip.open if out.endswith(".gz") else open
    with opener(out, "wt") as f:
        for r in recs:
            if set(r["times"]) != set(Variants(r["n"], r["prec"])):
                s = {k: r[k] for k in ("prec", "n", "batch", "real")}
                r = measure_shape(s, iters)
                n_new += 1
            f.write(json.dumps(r) + "\n")
    return n_new


DEFAULT_DATA = os.path.join(HERE, "wisdom", "planner_data.jsonl.gz")


def load_records(path: str = DEFAULT_DATA) -> list[dict]:
    import gzip
    opener = gzip.open if path.endswith(".gz") else open
    with opener(path, "rt") as f:
        return [json.loads(line) for line in f if line.strip()]


# ---------------------------------------------------------------- dataset

def design(records: list[dict]):
    """X (rows x D raw features), y (log ns per element), owner shape index,
    and the token of each row.  Variants without features (the L2-pipelined
    two-pass, an autotuner candidate only) are left out, as plan creation
    leaves them out of the model's candidates."""
    X, y, owner, toks = [], [], [], []
    for i, r in enumerate(records):
        for tok, ms in r["times"].items():
            try:
                x = features(r["prec"], r["n"], r["batch"], 1, r["real"], tok)
            except ErrInvalidArgument:
                continue
            X.append(x)
            y.append(math.log(ms * 1e6 / (r["n"] * r["batch"])))
            owner.append(i)
            toks.append(tok)
    return np.array(X, np.float32), np.array(y, np.float32), np.array(owner), toks


class Model:
    def __init__(self, params: np.ndarray, norm: np.ndarray):
        self.params = np.ascontiguousarray(params, np.float32)
        self.norm = np.ascontiguousarray(norm, np.float32)

    @staticmethod
    def norm_from(X: np.ndarray, y: np.ndarray) -> np.ndarray:
        mu = X.mean(0)
        sd = X.std(0)
        sd[sd < 1e-3] = 1.0
        return np.concatenate([mu, sd, [y.mean(), max(float(y.std()), 1e-3)]]).astype(np.float32)

    def standardize(self, X):
        d = X.shape[1]
        return ((X - self.norm[:d]) / self.norm[d:2 * d]).astype(np.float32)

    def save(self, path: str) -> None:
        d, h, _ = sizes()
        with open(path, "wb") as f:
            f.write(b"GFMLP1\0\0" + struct.pack("<ii", d, h))
            f.write(self.params.astype("<f4").tobytes())
            f.write(self.norm.astype("<f4").tobytes())

    @staticmethod
    def load(path: str) -> "Model":
        d, h, n = sizes()
        raw = open(path, "rb").read()
        assert raw[:8] == b"GFMLP1\0\0" and struct.unpack("<ii", raw[8:16]) == (d, h)
        v = np.frombuffer(raw[16:], "<f4")
        return Model(v[:n].copy(), v[n:n + 2 * d + 2].copy())

    def install(self) -> None:
        check(lib().gfft_planner_set_model(self.params.ctypes.data_as(ctypes.c_void_p),
                                           self.norm.ctypes.data_as(ctypes.c_void_p)))

    def predict(self, X: np.ndarray) -> np.ndarray:
        """Standardized predictions through gfft_mlp_forward (GPU)."""
        import torch
        xs = torch.from_numpy(self.standardize(X)).cuda()
        p = torch.from_numpy(self.params).cuda()
        out = torch.empty(xs.shape[0], dtype=torch.float32, device="cuda")
        check(lib().gfft_mlp_forward(p.data_ptr(), xs.data_ptr(), xs.shape[0], out.data_ptr(), None))
        torch.cuda.synchronize()
        return out.cpu().numpy()


def train(X: np.ndarray, y: np.ndarray, steps: int = 40000, batch: int = 64, lr: float = 2e-3, seed: int = 0,
          chunk: int = 1000, log=None) -> Model:
    """Adam on the GPU through gfft_mlp_train, cosine-decayed learning rate
    over launches of `chunk` steps; returns the trained model."""
    import torch
    norm = Model.norm_from(X, y)
    m = Model(init_params(seed), norm)
    xs = torch.from_numpy(m.standardize(X)).cuda()
    ys = torch.from_numpy(((y - norm[-2]) / norm[-1]).astype(np.float32)).cuda()
    p = torch.from_numpy(m.params.copy()).cuda()
    am = torch.zeros_like(p)
    av = torch.zeros_like(p)
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    done = 0
    while done < steps:
        k = min(chunk, steps - done)
        rate = lr * 0.5 * (1 + math.cos(math.pi * done / steps))
        check(lib().gfft_mlp_train(p.data_ptr(), am.data_ptr(), av.data_ptr(), xs.data_ptr(), ys.data_ptr(),
                                   xs.shape[0], k, batch, ctypes.c_float(rate), seed, done, loss.data_ptr(), None))
        done += k
        if log is not None:
            log(done, float(loss.item()))
    torch.cuda.synchronize()
    m.params = p.cpu().numpy()
    return m


# ---------------------------------------------------------------- evaluation

def regret_stats(records: list[dict], choose) -> dict:
    """choose(i, record) -> token; regret = t(chosen) / min t, per shape."""
    r = []
    for i, rec in enumerate(records):
        t = rec["times"]
        tok = choose(i, rec)
        r.append(t[tok] / min(t.values()) if tok in t else float("nan"))
    r = np.array(r)
    ok = r[np.isfinite(r)]
    return {"shapes": len(records), "mean": float(ok.mean()), "geomean": float(np.exp(np.log(ok).mean())),
            "median": float(np.median(ok)), "p90": float(np.percentile(ok, 90)), "max": float(ok.max()),
            "optimal": float(np.mean(ok <= 1.0 + 1e-9)), "missing": int(np.sum(~np.isfinite(r)))}


def learned_choices(model: Model, records: list[dict], predict=None) -> list[str]:
    X, _, owner, toks = design(records)
    pred = (predict or model.predict)(X)
    best = {}
    for j, i in enumerate(owner):
        if i not in best or pred[j] < pred[best[i]]:
            best[i] = j
    return [toks[best[i]] for i in range(len(records))]


def exercise(iters: int = 10) -> list[dict]:
    """The planner's exercise shapes end to end (device-resident data, one
    forward per step), planned three ways: size-class rules (empty wisdom,
    PlannerEstimate), the learned model (empty wisdom, PlannerLearned) and
    exhaustive measurement (PlannerMeasure: every variant timed at plan
    creation).  Bytes: the tensor's input and output once per transform."""
    import torch
    from .nd import NewPlan2D, NewPlanReal3D
    from .plan import PlannerEstimate, PlannerLearned, PlannerMeasure
    saved = ExportWisdomToString()
    out = []
    try:
        for planner, label in ((PlannerEstimate, "size_class_rules"), (PlannerLearned, "learned"),
                               (PlannerMeasure, "exhaustive")):
            ClearWisdom()
            # Plan2D complex64 4096 x 4096, batch 8
            o = PlanOptions(Planner=planner, Batch=8)
            x = torch.randn(8 * 4096 * 4096, dtype=torch.complex64, device="cuda")
            y = torch.empty_like(x)
            with NewPlan2D(4096, 4096, opts=o) as p:
                ms = _median_ms(lambda: p.Forward(y, x), iters)
            out.append({"shape": "Plan2D c64 4096x4096 batch 8", "planner": label, "ms": ms,
                        "GB/s": 2 * x.numel() * 8 / ms / 1e6})
            del x, y
            # PlanReal3D float32 256^3 (R2C)
            xr = torch.randn(256 ** 3, dtype=torch.float32, device="cuda")
            X = torch.empty(256 * 256 * 129, dtype=torch.complex64, device="cuda")
            with NewPlanReal3D(256, 256, 256, opts=PlanOptions(Planner=planner)) as p:
                ms = _median_ms(lambda: p.Forward(X, xr), iters)
            out.append({"shape": "PlanReal3D f32 256^3 R2C", "planner": label, "ms": ms,
                        "GB/s": (xr.numel() * 4 + X.numel() * 8) / ms / 1e6})
            # strided c64 column FFT: 4096 columns of length 1024 at stride 4096
            xs = torch.randn(1024 * 4096, dtype=torch.complex64, device="cuda")
            ys = torch.empty_like(xs)
            with Plan(1024, COMPLEX64, PlanOptions(Planner=planner)) as p:
                ms = _median_ms(lambda: p.StridedBatch(ys, xs, count=4096, stride=4096, dist=1), iters)
            out.append({"shape": "strided c64 N=1024 stride 4096 x 4096 columns", "planner": label, "ms": ms,
                        "GB/s": 2 * xs.numel() * 8 / ms / 1e6})
    finally:
        ClearWisdom()
        ImportWisdomFromString(saved)
    return out


def split(records: list[dict]):
    return records[:TRAIN_SHAPES], records[TRAIN_SHAPES:TRAIN_SHAPES + HELD_OUT_SHAPES]


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m algofft.planner")
    sub = ap.add_subparsers(dest="cmd", required=True)
    c = sub.add_parser("collect")
    c.add_argument("--count", type=int, default=TRAIN_SHAPES + HELD_OUT_SHAPES)
    c.add_argument("--seed", type=int, default=2024)
    c.add_argument("--iters", type=int, default=3)
    c.add_argument("--out", required=True)
    f = sub.add_parser("refresh")
    f.add_argument("--data", default=DEFAULT_DATA)
    f.add_argument("--iters", type=int, default=3)
    f.add_argument("--out", required=True)
    t = sub.add_parser("train")
    t.add_argument("--data", required=True)
    t.add_argument("--out", default=DEFAULT_MODEL)
    t.add_argument("--steps", type=int, default=40000)
    t.add_argument("--seed", type=int, default=0)
    r = sub.add_parser("report")
    r.add_argument("--data", default=DEFAULT_DATA)
    r.add_argument("--model", default=DEFAULT_MODEL)
    r.add_argument("--exercise", action="store_true", help="also time the exercise shapes")
    a = ap.parse_args(argv)
    if a.cmd == "collect":
        collect(a.count, a.seed, a.out, a.iters)
    elif a.cmd == "refresh":
        print(f"re-timed {refresh(a.data, a.out, a.iters)} shapes", file=sys.stderr)
    elif a.cmd == "train":
        tr, _ = split(load_records(a.data))
        X, y, _, _ = design(tr)
        m = train(X, y, steps=a.steps, seed=a.seed,
                  log=lambda s, l: print(json.dumps({"step": s, "loss": l}), file=sys.stderr, flush=True))
        m.save(a.out)
    else:
        m = Model.load(a.model)
        tr, te = split(load_records(a.data))
        rep = {}
        for name, recs in (("train", tr), ("held_out", te)):
            ch = learned_choices(m, recs)
            rep[name] = {"learned": regret_stats(recs, lambda i, rec: ch[i]),
                         "size_class_rules": regret_stats(recs, lambda i, rec: rec["default"])}
        if a.exercise:
            m.install()
            rep["exercise"] = exercise()
        print(json.dumps(rep, indent=1))
    return 0


if __name__ == "__main__":
    sys.exit(main())
