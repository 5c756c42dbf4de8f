"""Shared numerics for the parity tests."""
import math

import numpy as np


def rel_l2(got, want) -> float:
    got = np.asarray(got, dtype=np.complex128).ravel()
    want = np.asarray(want, dtype=np.complex128).ravel()
    den = np.linalg.norm(want)
    if den == 0:
        return float(np.linalg.norm(got))
    return float(np.linalg.norm(got - want) / den)


def tol_c2c(n: int, c128: bool) -> float:
    """Stated tolerance on relative L2 error against the FP64 oracle:
    1e-6*log2(N) for complex64, 1e-13*log2(N) for complex128 (N >= 2)."""
    lg = max(1.0, math.log2(max(n, 2)))
    return (1e-13 if c128 else 1e-6) * lg


def seeded_complex(n_total: int, seed: int, dtype=np.complex64, dist="normal") -> np.ndarray:
    """Seeded inputs; 'normal' = re, im i.i.d. N(0,1); 'uniform' = U[-1,1)."""
    rng = np.random.default_rng(seed)
    if dist == "normal":
        re = rng.standard_normal(n_total)
        im = rng.standard_normal(n_total)
    else:
        re = rng.uniform(-1.0, 1.0, n_total)
        im = rng.uniform(-1.0, 1.0, n_total)
    return (re + 1j * im).astype(dtype)
